// qs_watchdog.cu - self-test of the fused kernels' bounded waits.
//
// Every wait of the tensor-core kernels on an mbarrier (qs_tile::mbar_wait)
// gives up after a time limit, sets the error word that qs_plan_status reads,
// and lets the kernel return, so that a wait that can never end costs a
// bounded time and leaves the context usable.  qs_watchdog_selftest runs that
// helper on an mbarrier that nothing arrives on, with a caller-chosen limit,
// and reports through the same word: a test can make a wait run out without
// any GPU fault or hang.
#include "qs_common.cuh"
#include "qs_tile_core.cuh"

namespace {

__global__ void k_watchdog_selftest(int *err, unsigned long long limit_ns)
{
    __shared__ uint64_t mbar;
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(qs_tile::smem_u32(&mbar)), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;");
    }
    __syncthreads();
    // nothing arrives on this barrier: phase 0 never completes
    const bool ok = qs_tile::mbar_wait(qs_tile::smem_u32(&mbar), 0, limit_ns);
    if (!ok && threadIdx.x == 0) atomicExch(err, 1);
}

}  // namespace

extern "C" int qs_watchdog_selftest(qs_state *s, unsigned wait_us)
{
    int r = qs_check_state(s);
    if (r) return r;
    if (wait_us == 0 || wait_us > 2000000u)
        return qs_fail(QS_ERR_ARG, "qs_watchdog_selftest: wait of 1 us .. 2 s");
    const size_t kFlagOff = 64 * 1024 + 192;       // the word qs_plan_status reads
    int *flag = reinterpret_cast<int *>(static_cast<char *>(s->scratch) + kFlagOff);
    QS_CUDA_TRY(cudaMemsetAsync(flag, 0, sizeof(int), s->stream));
    k_watchdog_selftest<<<1, 32, 0, s->stream>>>(flag, 1000ull * wait_us);
    QS_LAUNCH_CHECK("k_watchdog_selftest");
    return QS_OK;
}
