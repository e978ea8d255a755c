/* Force-included when compiling the reference's unmodified sources with CUDA 12.9.
 *
 * operatorsCommunity.h:43 calls thrust::make_tuple<int, int, unsigned>(...) with an lvalue
 * `unsigned` argument. In CCCL 2.x thrust::make_tuple is cuda::std::make_tuple, whose
 * parameters are forwarding references, so an explicit `unsigned` template argument turns
 * the parameter into `unsigned&&` and the call no longer compiles. This overload accepts
 * explicit element types with deduced argument types and builds the same tuple the
 * CUDA 10.2 Thrust the reference was written for would have built. It changes no
 * behaviour of the reference code. */
#pragma once
#include <thrust/tuple.h>

namespace thrust {
template <class T0, class T1, class T2, class A0, class A1, class A2>
__host__ __device__ inline ::cuda::std::tuple<T0, T1, T2> make_tuple(A0&& a0, A1&& a1, A2&& a2) {
  return ::cuda::std::tuple<T0, T1, T2>(static_cast<T0>(a0), static_cast<T1>(a1), static_cast<T2>(a2));
}
}  // namespace thrust
