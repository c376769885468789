// walk32.cu -- FP32 walk (placeholder until the fast kernel lands): refuses.
#include "internal.h"

namespace gg
{
cudaError_t walk32_stage(gpugrav_ctx *c, const WalkConst &wc)
{
  (void)c;
  (void)wc;
  return cudaErrorNotSupported;
}
cudaError_t layout32_stage(gpugrav_ctx *c)
{
  (void)c;
  return cudaErrorNotSupported;
}
}  // namespace gg
