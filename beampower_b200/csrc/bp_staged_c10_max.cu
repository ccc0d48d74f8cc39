// Staged kernel variants of config 10, max/argmax reduction.
#include "bp_staged.cuh"

namespace bp_host {
template int launch_window_c<10, true>(int, bool, int, const bp::LaunchArgs&, bool,
                                             long long, int, cudaStream_t);
}  // namespace bp_host
