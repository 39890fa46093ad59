// Registry of the device allocations libttcuda owns.  Every kernel descriptor built by a
// plan is checked against it on the host before anything is launched, so an addressing
// mistake in a descriptor raises TTC_EINTERNAL instead of touching memory it does not own.
#pragma once
#include <cstddef>
#include <cstdint>
#include <string>

namespace ttc {

void region_add(const void* p, size_t bytes);
void region_remove(const void* p);
// Throws Error(TTC_EINTERNAL, what) unless [p, p + bytes) lies inside one registered region.
void region_check(const void* p, size_t bytes, const char* what);
// Extent (in elements) of an index map sum_i idx_i * stride_i with idx_i < ext_i (strides >= 0).
long long span_elems(const long long* ext, const long long* stride, int n);

}  // namespace ttc
