// Fused-scan kernels of nbasis group 3 (rr_fused.cuh).
#include "rr_fused.cuh"

namespace rr {

int fused_group_3(bool exty, int zt, int bgroup, const rr_scan_targets* targets,
                   const rr_scan_template* templates, const int* pick, int npick, int* counter,
                   int* resweep, int* status, bool overlap, cudaStream_t stream) {
  return exty ? launch_group<3, true>(zt, bgroup, targets, templates, pick, npick, counter, resweep,
                                        status, overlap, stream)
              : launch_group<3, false>(zt, bgroup, targets, templates, pick, npick, counter, resweep,
                                         status, overlap, stream);
}

}  // namespace rr
