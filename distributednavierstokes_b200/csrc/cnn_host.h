// Host-side facts of a closure that the FV context needs before it reuses
// a CUDA graph captured around the closure's inference (C++ linkage, not
// part of the C ABI).
#pragma once

struct dnsb_cnn;

namespace dnsb_internal {

// a number unique to this closure among all created in the process: every
// buffer the inference launches read or write lives as long as the closure
unsigned long long cnn_serial(const dnsb_cnn *c);
// per-launch event timing on (launches then record events, which a
// captured graph must not hold)
bool cnn_profiling(const dnsb_cnn *c);

}  // namespace dnsb_internal
