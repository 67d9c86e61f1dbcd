// stream_copy.cuh -- asynchronous global -> shared copies of data read once
// (cp.async), under an L2 policy that evicts it first: the streamed
// operator rows pass through L2 while the vector they are applied to, which
// every row gathers from, stays resident.
#pragma once

namespace rbfb {

__device__ __forceinline__ unsigned long long evict_first_policy() {
    unsigned long long pol;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;\n" : "=l"(pol));
    return pol;
}
// BYTES = 16: .cg, to shared memory through L2 only (both addresses 16-byte
// aligned); 4 or 8: .ca.
template <int BYTES>
__device__ __forceinline__ void cp_async_stream(void* dst, const void* src,
                                                unsigned long long pol) {
    if constexpr (BYTES == 16)
        asm volatile("cp.async.cg.shared.global.L2::cache_hint [%0], [%1], 16, %2;\n" ::"r"(
                         (unsigned)__cvta_generic_to_shared(dst)),
                     "l"(src), "l"(pol)
                     : "memory");
    else
        asm volatile("cp.async.ca.shared.global.L2::cache_hint [%0], [%1], %2, %3;\n" ::"r"(
                         (unsigned)__cvta_generic_to_shared(dst)),
                     "l"(src), "n"(BYTES), "l"(pol)
                     : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}
template <int PENDING>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(PENDING) : "memory");
}
// Waits until at most `pending` (0..3; a constant once the caller's loop is
// unrolled) of this thread's copy groups are still in flight.
__device__ __forceinline__ void cp_async_wait_pending(int pending) {
    switch (pending) {
        case 0: cp_async_wait<0>(); break;
        case 1: cp_async_wait<1>(); break;
        case 2: cp_async_wait<2>(); break;
        default: cp_async_wait<3>(); break;
    }
}

}  // namespace rbfb
