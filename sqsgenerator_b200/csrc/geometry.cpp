// Host precompute of the SQS optimisation: geometry, coordination shells, prefactors, pair list and
// the sort of sites by sublattice. Runs once per job on the CPU, before the device loop.
//
// Each function restates the reference function named beside it (dgehringer/sqsgenerator 0.5.6,
// paths relative to its repository root) in the job's floating type T with the same operation order,
// so shell assignment, prefactors and pair lists match the reference's.

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <map>
#include <set>
#include <stdexcept>
#include <vector>

#include "sqsg_internal.h"

namespace sqsg {

template <class T> static bool is_close(T a, T b, T atol, T rtol) {
  // core/helpers/numeric.h:11-14
  return std::abs(a - b) <= (atol + rtol * std::abs(b));
}

// core/structure.h:335-366. The diagonal scale matrix is inverted like Eigen's 3x3 cofactor inverse
// (cofactor * (1/det)).
template <class T>
static void supercell(const T* lattice, const T* frac, const uint8_t* species, uint32_t n, uint32_t a,
                      uint32_t b, uint32_t c, T* lattice_out, T* frac_out, uint8_t* species_out) {
  const T da = static_cast<T>(a), db = static_cast<T>(b), dc = static_cast<T>(c);
  const T det = (db * dc) * da;
  const T invdet = T(1) / det;
  const T inv[3] = {(db * dc) * invdet, (da * dc) * invdet, (da * db) * invdet};
  std::vector<T> scaled(static_cast<size_t>(n) * 3);
  for (uint32_t s = 0; s < n; ++s)
    for (int k = 0; k < 3; ++k) scaled[3 * s + k] = frac[3 * s + k] * inv[k];
  size_t idx = 0;
  for (uint32_t i = 0; i < a; ++i)
    for (uint32_t j = 0; j < b; ++j)
      for (uint32_t k = 0; k < c; ++k) {
        const T tr[3] = {static_cast<T>(i) * inv[0], static_cast<T>(j) * inv[1], static_cast<T>(k) * inv[2]};
        for (uint32_t s = 0; s < n; ++s, ++idx) {
          for (int d = 0; d < 3; ++d) frac_out[3 * idx + d] = tr[d] + scaled[3 * s + d];
          species_out[idx] = species[s];
        }
      }
  const T sc[3] = {da, db, dc};
  for (int r = 0; r < 3; ++r)
    for (int col = 0; col < 3; ++col) lattice_out[3 * r + col] = lattice[3 * r + col] * sc[col];
}

// core/structure.h:35-69 — per pair the minimum norm over the 27 images; each inner product of
// three terms is summed x0 + (x1 + x2).
template <class T> static void distance_matrix(const T* lattice, const T* frac, uint32_t n, T* out) {
  std::vector<T> cart(static_cast<size_t>(n) * 3);
  for (uint32_t i = 0; i < n; ++i)
    for (int j = 0; j < 3; ++j) {
      T x0 = frac[3 * i + 0] * lattice[0 * 3 + j];
      T x1 = frac[3 * i + 1] * lattice[1 * 3 + j];
      T x2 = frac[3 * i + 2] * lattice[2 * 3 + j];
      cart[3 * i + j] = x0 + (x1 + x2);
    }
  T shifts[27][3];
  int t = 0;
  for (int u = -1; u <= 1; ++u)
    for (int v = -1; v <= 1; ++v)
      for (int w = -1; w <= 1; ++w, ++t)
        for (int d = 0; d < 3; ++d)
          shifts[t][d] = (static_cast<T>(u) * lattice[0 * 3 + d] + static_cast<T>(v) * lattice[1 * 3 + d]) +
                         static_cast<T>(w) * lattice[2 * 3 + d];
  const T big = std::numeric_limits<T>::max();
  for (size_t k = 0; k < static_cast<size_t>(n) * n; ++k) out[k] = big;
  for (uint32_t i = 0; i < n; ++i)
    for (uint32_t j = i; j < n; ++j) {
      T best = big;
      for (int s = 0; s < 27; ++s) {
        T d0 = cart[3 * i + 0] - (shifts[s][0] + cart[3 * j + 0]);
        T d1 = cart[3 * i + 1] - (shifts[s][1] + cart[3 * j + 1]);
        T d2 = cart[3 * i + 2] - (shifts[s][2] + cart[3 * j + 2]);
        T nrm = std::abs(std::sqrt(d0 * d0 + (d1 * d1 + d2 * d2)));
        if (nrm < best) best = nrm;
      }
      out[static_cast<size_t>(i) * n + j] = best;
      out[static_cast<size_t>(j) * n + i] = best;
    }
}

// core/structure.h:71-100
template <class T>
static void shell_matrix(const T* dist, uint32_t n, const T* radii, uint32_t n_radii, T atol, T rtol,
                         uint32_t* out) {
  auto find_shell = [&](T d) -> uint32_t {
    if (d < 0) throw std::out_of_range("Invalid distance matrix input");
    if (is_close<T>(d, T(0.0), atol, rtol)) return 0;
    for (uint32_t i = 0; i + 1 < n_radii; i++) {
      T lb = radii[i], up = radii[i + 1];
      if ((is_close(d, lb, atol, rtol) || d > lb) && (is_close(d, up, atol, rtol) || up > d)) return i + 1;
    }
    return n_radii;
  };
  for (uint32_t i = 0; i < n; ++i) {
    out[static_cast<size_t>(i) * n + i] = 0;
    for (uint32_t j = i + 1; j < n; ++j) {
      uint32_t s = find_shell(dist[static_cast<size_t>(i) * n + j]);
      out[static_cast<size_t>(i) * n + j] = s;
      out[static_cast<size_t>(j) * n + i] = s;
    }
  }
}

// core/structure.h:195-207 — unique sorted distances, near-equal neighbours merged to their mean.
template <class T>
static std::vector<T> distances_naive(const T* dist, uint32_t n, T atol, T rtol) {
  std::set<T> uniq(dist, dist + static_cast<size_t>(n) * n);
  std::vector<T> vec{T(0)};
  for (T d : uniq) {
    if (is_close(vec.back(), d, atol, rtol))
      vec.back() = static_cast<T>(0.5 * (d + vec.back()));
    else
      vec.push_back(d);
  }
  return vec;
}

// core/structure.h:209-258 — histogram peak detection.
template <class T>
static std::vector<T> distances_histogram(const T* dist, uint32_t n, T bin_width, T peak_isolation) {
  std::vector<T> d;
  for (size_t k = 0; k < static_cast<size_t>(n) * n; ++k)
    if (dist[k] > 0.0 && !is_close<T>(dist[k], T(0.0), T(1.0e-5), T(1.0e-3))) d.push_back(dist[k]);
  if (d.empty()) throw std::invalid_argument("no non-zero distances");
  std::sort(d.begin(), d.end());
  T mn = d.front(), mx = d.back();
  size_t num_edges = static_cast<size_t>((mx - mn) / bin_width) + 2;
  std::vector<T> edges(num_edges);
  for (size_t i = 0; i < num_edges; i++) edges[i] = mn + static_cast<T>(i) * bin_width;
  if (edges.size() < 10)
    throw std::invalid_argument("Not enough edges to create a histogram, please increase the bin width");
  std::map<size_t, std::vector<T>> freqs{{0, {}}};
  size_t index = 0, bin = 0;
  while (index < d.size() && bin < num_edges - 1) {
    T lower = edges[bin], upper = edges[bin + 1], value = d[index];
    if (lower <= value && value < upper) {
      freqs[bin].push_back(value);
      ++index;
    } else {
      freqs[++bin] = std::vector<T>{};
    }
  }
  auto get = [&](long long i) -> std::vector<T> {
    if (i < 0) return {};
    auto it = freqs.find(static_cast<size_t>(i));
    return it == freqs.end() ? std::vector<T>{} : it->second;
  };
  std::vector<T> shells;
  for (long long i = 0; i <= static_cast<long long>(num_edges); i++) {
    auto prev = get(i - 1), f = get(i), next = get(i + 1);
    auto threshold = static_cast<size_t>((1.0 - peak_isolation) * static_cast<T>(f.size()));
    if (threshold > prev.size() && threshold > next.size()) shells.push_back(*std::max_element(f.begin(), f.end()));
  }
  if (shells.empty()) throw std::invalid_argument("no coordination shell peaks found");
  if (shells.front() != 0.0 && !is_close<T>(shells.front(), T(0.0), T(1.0e-5), T(1.0e-3)))
    shells.insert(shells.begin(), T(0.0));
  return shells;
}

// core/structure.h:136-192. The per-shell site count is stored back into an integer counter, so
// count/N is truncated before it becomes M_i.
template <class T>
static void prefactors(const uint32_t* shells, uint32_t n, const uint32_t* shell_ids, uint32_t n_shells,
                       const uint8_t* species, T* out) {
  if (n_shells == 0) throw std::out_of_range("no coordination shells selected");
  std::map<uint32_t, uint64_t> neighbors;
  for (size_t k = 0; k < static_cast<size_t>(n) * n; ++k) neighbors[shells[k]]++;
  for (auto& [shell, count] : neighbors) {
    T per = static_cast<T>(count) / static_cast<T>(n);
    count = static_cast<uint64_t>(per);
  }
  std::map<uint8_t, uint64_t> hist;
  for (uint32_t i = 0; i < n; ++i) hist[species[i]]++;
  std::vector<uint8_t> zs;
  for (auto& [z, c] : hist) zs.push_back(z);
  const size_t K = zs.size();
  for (uint32_t s = 0; s < n_shells; s++) {
    auto it = neighbors.find(shell_ids[s]);
    uint64_t nc = it == neighbors.end() ? 0 : it->second;
    for (size_t a = 0; a < K; a++)
      for (size_t b = a; b < K; b++) {
        T p = T(0);
        if (nc > 0) {
          T M = static_cast<T>(nc);
          T xa = static_cast<T>(hist[zs[a]]) / static_cast<T>(n);
          T xb = static_cast<T>(hist[zs[b]]) / static_cast<T>(n);
          p = T(1.0) / (M * xa * xb * static_cast<T>(n));
        }
        out[(s * K + a) * K + b] = p;
        out[(s * K + b) * K + a] = p;
      }
  }
}

}  // namespace sqsg

using namespace sqsg;

template <class T> static sqsg_status copy_out(const std::vector<T>& v, void* out, uint32_t* n_out) {
  uint32_t cap = *n_out;
  *n_out = static_cast<uint32_t>(v.size());
  if (v.size() > cap) {
    set_error("output capacity too small");
    return SQSG_ERR_CAPACITY;
  }
  std::memcpy(out, v.data(), v.size() * sizeof(T));
  return SQSG_OK;
}

extern "C" {

sqsg_status sqsg_supercell(int prec, const void* lattice, const void* frac, const uint8_t* species, uint32_t n,
                           uint32_t a, uint32_t b, uint32_t c, void* lattice_out, void* frac_out,
                           uint8_t* species_out) {
  return guarded([&] {
    if (a == 0 || b == 0 || c == 0) throw std::invalid_argument("There must be at least one copy in each direction");
    if (!lattice || !frac || !species || !lattice_out || !frac_out || !species_out)
      throw std::invalid_argument("null pointer");
    if (prec == SQSG_PREC_DOUBLE)
      supercell(static_cast<const double*>(lattice), static_cast<const double*>(frac), species, n, a, b, c,
                static_cast<double*>(lattice_out), static_cast<double*>(frac_out), species_out);
    else
      supercell(static_cast<const float*>(lattice), static_cast<const float*>(frac), species, n, a, b, c,
                static_cast<float*>(lattice_out), static_cast<float*>(frac_out), species_out);
  });
}

sqsg_status sqsg_distance_matrix(int prec, const void* lattice, const void* frac, uint32_t n, void* out) {
  return guarded([&] {
    if (!lattice || !frac || !out) throw std::invalid_argument("null pointer");
    if (prec == SQSG_PREC_DOUBLE)
      distance_matrix(static_cast<const double*>(lattice), static_cast<const double*>(frac), n,
                      static_cast<double*>(out));
    else
      distance_matrix(static_cast<const float*>(lattice), static_cast<const float*>(frac), n,
                      static_cast<float*>(out));
  });
}

sqsg_status sqsg_shell_matrix(int prec, const void* distances, uint32_t n, const void* radii, uint32_t n_radii,
                              double atol, double rtol, uint32_t* out) {
  return guarded([&] {
    if (!distances || !radii || !out) throw std::invalid_argument("null pointer");
    if (prec == SQSG_PREC_DOUBLE)
      shell_matrix(static_cast<const double*>(distances), n, static_cast<const double*>(radii), n_radii, atol,
                   rtol, out);
    else
      shell_matrix(static_cast<const float*>(distances), n, static_cast<const float*>(radii), n_radii,
                   static_cast<float>(atol), static_cast<float>(rtol), out);
  });
}

sqsg_status sqsg_distances_naive(int prec, const void* distances, uint32_t n, double atol, double rtol, void* out,
                                 uint32_t* n_out) {
  sqsg_status st = SQSG_OK;
  sqsg_status g = guarded([&] {
    if (!distances || !out || !n_out) throw std::invalid_argument("null pointer");
    if (prec == SQSG_PREC_DOUBLE)
      st = copy_out(distances_naive(static_cast<const double*>(distances), n, atol, rtol), out, n_out);
    else
      st = copy_out(distances_naive(static_cast<const float*>(distances), n, static_cast<float>(atol),
                                    static_cast<float>(rtol)),
                    out, n_out);
  });
  return g != SQSG_OK ? g : st;
}

sqsg_status sqsg_distances_histogram(int prec, const void* distances, uint32_t n, double bin_width,
                                     double peak_isolation, void* out, uint32_t* n_out) {
  sqsg_status st = SQSG_OK;
  sqsg_status g = guarded([&] {
    if (!distances || !out || !n_out) throw std::invalid_argument("null pointer");
    if (prec == SQSG_PREC_DOUBLE)
      st = copy_out(distances_histogram(static_cast<const double*>(distances), n, bin_width, peak_isolation), out,
                    n_out);
    else
      st = copy_out(distances_histogram(static_cast<const float*>(distances), n, static_cast<float>(bin_width),
                                        static_cast<float>(peak_isolation)),
                    out, n_out);
  });
  return g != SQSG_OK ? g : st;
}

sqsg_status sqsg_prefactors(int prec, const uint32_t* shells, uint32_t n, const uint32_t* shell_ids,
                            uint32_t n_shells, const uint8_t* species, void* out) {
  return guarded([&] {
    if (!shells || !shell_ids || !species || !out) throw std::invalid_argument("null pointer");
    if (prec == SQSG_PREC_DOUBLE)
      prefactors(shells, n, shell_ids, n_shells, species, static_cast<double*>(out));
    else
      prefactors(shells, n, shell_ids, n_shells, species, static_cast<float*>(out));
  });
}

sqsg_status sqsg_pairs(const uint32_t* shells, uint32_t n, const uint32_t* shell_ids, uint32_t n_shells,
                       uint32_t* pairs_out, uint32_t* n_pairs) {
  sqsg_status st = SQSG_OK;
  sqsg_status g = guarded([&] {
    if (!shells || !shell_ids || !n_pairs) throw std::invalid_argument("null pointer");
    std::map<uint32_t, uint32_t> index;  // make_index_mapping over the weighted shells
    std::vector<uint32_t> ids(shell_ids, shell_ids + n_shells);
    std::sort(ids.begin(), ids.end());
    for (uint32_t k = 0; k < ids.size(); ++k) index[ids[k]] = k;
    uint64_t cap = *n_pairs, count = 0;
    for (uint32_t i = 0; i < n; ++i)
      for (uint32_t j = i + 1; j < n; ++j) {
        auto it = index.find(shells[static_cast<size_t>(i) * n + j]);
        if (it == index.end()) continue;
        if (count < cap && pairs_out) {
          pairs_out[3 * count + 0] = i;
          pairs_out[3 * count + 1] = j;
          pairs_out[3 * count + 2] = it->second;
        }
        ++count;
      }
    *n_pairs = static_cast<uint32_t>(count);
    if (count > cap) {
      set_error("pair capacity too small");
      st = SQSG_ERR_CAPACITY;
    }
  });
  return g != SQSG_OK ? g : st;
}

// optimization::compute_shuffling_bounds (core/optimization.h:35-72): the same std::sort call
// (libstdc++, not stable) with the same comparator on the same input, so equal keys land in the
// reference's order.
sqsg_status sqsg_sort_by_sublattice(const uint32_t* sublattice_of_site, uint32_t n, uint32_t n_sublattices,
                                    uint32_t* sort_order, uint32_t* windows, uint32_t* n_windows) {
  return guarded([&] {
    if (!sublattice_of_site || !sort_order || !windows || !n_windows) throw std::invalid_argument("null pointer");
    if (n == 0) throw std::invalid_argument("empty structure");
    struct Site {
      uint64_t index;
    };
    std::vector<Site> sites(n);
    for (uint32_t i = 0; i < n; ++i) sites[i].index = i;
    std::sort(sites.begin(), sites.end(), [&](const Site& a, const Site& b) {
      return sublattice_of_site[a.index] < sublattice_of_site[b.index];
    });
    std::vector<uint32_t> idx(n);
    for (uint32_t i = 0; i < n; ++i) {
      sort_order[i] = static_cast<uint32_t>(sites[i].index);
      idx[i] = sublattice_of_site[sites[i].index];
    }
    uint32_t cap = *n_windows, count = 0, lower = 0;
    auto push = [&](uint32_t lo, uint32_t hi) {
      if (count < cap) {
        windows[2 * count] = lo;
        windows[2 * count + 1] = hi;
      }
      ++count;
    };
    for (uint32_t i = 0; i < n; ++i) {
      if (idx[i] != idx[lower]) {
        push(lower, i);
        lower = i;
        if (idx[i] == n_sublattices) break;
      } else if (i == n - 1) {
        push(lower, i + 1);
      }
    }
    *n_windows = count;
    if (count > cap) throw std::length_error("window capacity too small");
  });
}

}  // extern "C"
