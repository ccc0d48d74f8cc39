// Staged kernel variants of config 9, full beams (no reduction).
#include "bp_staged.cuh"

namespace bp_host {
template int launch_window_c<9, false>(int, bool, int, const bp::LaunchArgs&, bool,
                                             long long, int, cudaStream_t);
}  // namespace bp_host
