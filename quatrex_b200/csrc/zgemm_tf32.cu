// Mixed-precision complex GEMM (3xTF32 split products on tcgen05) -- entry
// points; the kernel lands with the mixed-precision form.
#include "kernels.h"

bool tf32x3_supported(const GemmCall&) { return false; }

void launch_zgemm_tf32x3(const GemmCall&, cudaStream_t) {
  throw QtxError(QTX_E_UNSUPPORTED, "mixed-precision GEMM not available");
}
