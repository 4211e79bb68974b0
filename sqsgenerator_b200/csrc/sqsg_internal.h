// Internal declarations shared by the host precompute, the device engine and the C ABI.
#pragma once

#include <cstdint>
#include <exception>
#include <new>
#include <stdexcept>
#include <string>

#include "../../include/sqsgen_b200.h"

namespace sqsg {

void set_error(const std::string& msg);

// Process-wide options (sqsg_set_option / sqsg_get_option).
enum Option : int {
  kOptForceGeneral = 0,     // 1: every job takes the general pair-stream path
  kOptStageWaitNs = 1,      // bound of the device's staging wait in nanoseconds
  kOptDebugSkipStaging = 2, // debug: issue no staging copy, so that the bounded wait runs out
  kOptUseTuning = 3,        // 1: jobs take the measured launch choices of their bucket (tuning table)
  kOptDefaultCandidates = 4,  // candidate capacity of a job that leaves max_results at 0
  kOptRerunRecordBytes = 5,   // bytes of full records a re-run of an overflowed job may produce
  kOptRapidrand = 6,          // debug: random jobs follow the reference's seeded single-thread trajectory
  kOptServerFinalizers = 7,   // result-selection threads of a server created afterwards
  kOptBinaryFloyd = 8,        // 1: random windows of two species draw their minority sites (Floyd)
  kOptCount
};
long long option(Option o);

// Raises the dynamic shared-memory attribute of `kernel` on the current device to at least `bytes`
// (per device, never lowered, one mutex for every entry point). Returns the CUDA status as int.
int raise_dynamic_smem(const void* kernel, size_t bytes);

// An error raised by the CUDA runtime or a device-side status word.
struct cuda_error : std::runtime_error {
  using std::runtime_error::runtime_error;
};
struct unsupported_error : std::runtime_error {
  using std::runtime_error::runtime_error;
};
struct timeout_error : std::runtime_error {
  using std::runtime_error::runtime_error;
};


// Runs fn, translating C++ exceptions into an sqsg_status plus the thread's last-error message.
template <class Fn> sqsg_status guarded(Fn&& fn) {
  try {
    fn();
    return SQSG_OK;
  } catch (std::out_of_range const& e) {
    set_error(e.what());
    return SQSG_ERR_OUT_OF_RANGE;
  } catch (std::length_error const& e) {
    set_error(e.what());
    return SQSG_ERR_CAPACITY;
  } catch (std::invalid_argument const& e) {
    set_error(e.what());
    return SQSG_ERR_INVALID_ARGUMENT;
  } catch (unsupported_error const& e) {
    set_error(e.what());
    return SQSG_ERR_UNSUPPORTED;
  } catch (timeout_error const& e) {
    set_error(e.what());
    return SQSG_ERR_TIMEOUT;
  } catch (std::bad_alloc const&) {
    set_error("out of host memory");
    return SQSG_ERR_CAPACITY;
  } catch (std::exception const& e) {
    set_error(e.what());
    return SQSG_ERR_CUDA;
  }
}

}  // namespace sqsg
