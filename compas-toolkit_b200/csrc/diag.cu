// diag.cu — a kernel whose bounded device-side wait runs out, for tests of the failure channel.
//
// Kernels of this library never trap: a wait that gives up records STATUS_WAIT_TIMEOUT in the
// status word of the context the kernel was launched through and returns, and the host raises
// CompasException at the next synchronisation (the reference's device assertion traps instead,
// include/compas/core/assertion.h:24). The probe below waits, with the same bounded wait the
// tensor-core pipelines use, on a barrier that nothing arrives on, so the timeout path runs
// without an operation in flight that could be left half done.
#include "common.cuh"
#include "kernels.h"
#include "tc_common.cuh"

namespace compas {
namespace kernels {

__global__ void wait_probe_kernel(unsigned int* status, long long limit_cycles) {
    __shared__ uint64_t bar;
    if (threadIdx.x != 0) return;
    tc::mbar_init(&bar, 1);  // one arrival completes phase 0; none is made
    (void)tc::mbar_wait(&bar, 0, status, limit_cycles);
}

}  // namespace kernels

void launch_wait_probe(const CompasContext& ctx, long long limit_cycles) {
    if (limit_cycles < 0) COMPAS_ERROR("wait limit must be non-negative");
    DeviceGuard guard(ctx.device());
    kernels::wait_probe_kernel<<<1, 32, 0, ctx.stream()>>>(ctx.status_word(), limit_cycles);
    check_launch("wait_probe_kernel");
}

}  // namespace compas
