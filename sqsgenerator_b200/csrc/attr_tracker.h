// Per-(device, kernel) bookkeeping of the dynamic shared-memory attribute.
//
// cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, n) applies to the current
// device only, so a process that launches on two devices has to raise it on each. Every entry point
// goes through one tracker: one mutex, one record per (device, kernel), and the attribute is only
// ever raised, never lowered, so that a launch sized by one entry point is never invalidated by
// another. The tracker has no CUDA dependency of its own (the caller passes the setter), which lets
// a CPU test exercise the bookkeeping with a fake setter.
#pragma once

#include <cstddef>
#include <map>
#include <mutex>
#include <utility>

namespace sqsg {

class DynamicSmemTracker {
 public:
  // Calls set(bytes) when `bytes` is above what was set for (device, kernel) so far; returns the
  // setter's status (0 = success), or 0 when nothing had to be set.
  template <class Set> int raise(int device, const void* kernel, size_t bytes, Set&& set) {
    std::lock_guard<std::mutex> l(m_);
    size_t& cur = set_[{device, kernel}];
    if (bytes <= cur) return 0;
    const int err = set(bytes);
    if (err == 0) cur = bytes;
    return err;
  }
  size_t current(int device, const void* kernel) {
    std::lock_guard<std::mutex> l(m_);
    auto it = set_.find({device, kernel});
    return it == set_.end() ? 0 : it->second;
  }

 private:
  std::mutex m_;
  std::map<std::pair<int, const void*>, size_t> set_;
};

}  // namespace sqsg
