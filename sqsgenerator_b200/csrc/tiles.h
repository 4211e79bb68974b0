// Tile decomposition of a job's configuration range. A configuration depends only on the job and
// its id (random mode: a shuffle with words seeded by id; systematic mode: rank = id), so any
// decomposition evaluates the same configurations; tiles only shape the schedule.
//
// Tiles are guided: each takes about 1/2048 of what is left (large tiles first, then smaller ones
// toward the end, which evens out the finish across CTAs), with at least `floor` configurations
// per thread and at most max_per_thread (65,536 by default; the server caps tiles shorter so that
// SMs can change hands between jobs quickly).
#pragma once

#include <algorithm>
#include <cstdint>
#include <type_traits>

#include "engine.cuh"

namespace sqsg {

template <class Emit>
inline void for_each_tile(uint64_t first, uint64_t count, bool systematic, Emit&& emit,
                          uint64_t max_per_thread = 1u << 16) {
  if (count == 0) return;
  const uint64_t floor = std::max<uint64_t>(1, std::min<uint64_t>(16, count / (static_cast<uint64_t>(kBlock) * 8192)));
  uint64_t done = 0;
  while (done < count) {
    const uint64_t left = count - done;
    uint64_t cpt = (left + static_cast<uint64_t>(kBlock) * 2048 - 1) / (static_cast<uint64_t>(kBlock) * 2048);
    cpt = std::min<uint64_t>(std::max(cpt, floor), std::max<uint64_t>(1, max_per_thread));
    Tile t{};
    t.count = std::min<uint64_t>(cpt * kBlock, left);
    t.start = first + done + (systematic ? 1 : 0);
    if constexpr (std::is_same_v<decltype(emit(t)), bool>) {
      if (!emit(t)) return;  // the caller has seen enough tiles
    } else {
      emit(t);
    }
    done += t.count;
  }
}

}  // namespace sqsg
