// Forced into cuGriddingConvolution.cu only.  With CCCL 2.8 its unqualified
// inclusive_scan(device_vector<unsigned>::iterator..., thrust::plus<unsigned>)
// (cuGriddingConvolution.cu:374) is ambiguous between thrust:: and the
// cuda::std:: overload found by argument-dependent lookup.  A non-template
// overload in the caller's namespace is the exact match and forwards to
// thrust::inclusive_scan, which is what the reference meant to call.
#pragma once
#include <thrust/device_vector.h>
#include <thrust/functional.h>
#include <thrust/scan.h>
namespace Gadgetron {
using gb_ref_u32_iterator = thrust::device_vector<unsigned int>::iterator;
inline gb_ref_u32_iterator inclusive_scan(gb_ref_u32_iterator first, gb_ref_u32_iterator last,
                                          gb_ref_u32_iterator out, thrust::plus<unsigned int> op) {
    return thrust::inclusive_scan(first, last, out, op);
}
}  // namespace Gadgetron
