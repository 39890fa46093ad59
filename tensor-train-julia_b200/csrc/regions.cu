#include <map>
#include <mutex>

#include "common.cuh"
#include "regions.cuh"

namespace ttc {
namespace {
std::mutex g_mu;
std::map<uintptr_t, size_t>& regions() {
  static std::map<uintptr_t, size_t> m;
  return m;
}
}  // namespace

void region_add(const void* p, size_t bytes) {
  if (!p) return;
  std::lock_guard<std::mutex> l(g_mu);
  regions()[(uintptr_t)p] = bytes;
}

void region_remove(const void* p) {
  if (!p) return;
  std::lock_guard<std::mutex> l(g_mu);
  regions().erase((uintptr_t)p);
}

void region_check(const void* p, size_t bytes, const char* what) {
  if (bytes == 0) return;
  const uintptr_t a = (uintptr_t)p;
  std::lock_guard<std::mutex> l(g_mu);
  auto& m = regions();
  auto it = m.upper_bound(a);
  if (it != m.begin()) {
    --it;
    if (a >= it->first && a + bytes <= it->first + it->second) return;
  }
  throw Error(TTC_EINTERNAL, std::string("descriptor outside device allocations: ") + what);
}

long long span_elems(const long long* ext, const long long* stride, int n) {
  long long s = 0;
  for (int i = 0; i < n; ++i) {
    if (ext[i] <= 0) return 0;
    if (stride[i] < 0) throw Error(TTC_EINTERNAL, "negative stride in a descriptor");
    s += (ext[i] - 1) * stride[i];
  }
  return s + 1;
}

}  // namespace ttc
