// TEST ORACLE shim: C entry points over the reference's own rts/ops.cpp and
// rts/dependency.cpp (compiled unmodified from the reference tree by oracle/Makefile).
#include <ops.h>
#include <dependency.h>

#include <cstdint>
#include <vector>

extern "C" {

int ref_check_overlap(uintptr_t pa, size_t pitch_a, size_t width_a, size_t height_a, uintptr_t pb, size_t pitch_b,
                      size_t width_b, size_t height_b) {
  DataMap2D a(reinterpret_cast<void*>(pa), pitch_a, width_a, height_a);
  DataMap2D b(reinterpret_cast<void*>(pb), pitch_b, width_b, height_b);
  return a.checkOverlap(b) ? 1 : 0;
}

int ref_dependency_combine(int a, int b) { return (int)((dependency_t)a + (dependency_t)b); }

void* ref_table_create() { return new dependency_table(); }
void ref_table_destroy(void* t) { delete static_cast<dependency_table*>(t); }
void ref_table_update(void* t, long long from, long long to, int dep) {
  static_cast<dependency_table*>(t)->update(from, to, (dependency_t)dep);
}
int ref_table_lookup(void* t, long long from, long long to) {
  return (int)static_cast<dependency_table*>(t)->lookup(from, to);
}
long long ref_table_count_from(void* t, long long from) { return (long long)static_cast<dependency_table*>(t)->countDepFrom(from); }
long long ref_table_count_to(void* t, long long to) { return (long long)static_cast<dependency_table*>(t)->countDepTo(to); }
// fills out[] (capacity cap) with getDepFrom / getDepTo; returns the list length
long long ref_table_list(void* t, long long node, int to_side, long long* out, long long cap) {
  std::vector<int64_t> lis;
  if (to_side) static_cast<dependency_table*>(t)->getDepTo(node, lis);
  else static_cast<dependency_table*>(t)->getDepFrom(node, lis);
  for (size_t i = 0; i < lis.size() && (long long)i < cap; ++i) out[i] = lis[i];
  return (long long)lis.size();
}

}  // extern "C"
