// Cross-check shim -- TEST INFRASTRUCTURE ONLY.
//
// Exposes a few reference runtime functions, compiled straight from the
// reference sources by `make -C oracle ref`, through a C ABI so the tests can
// compare the oracle's restatements against them:
//   runtime::Date::{DateBuilder::Build, SplitDate}   (runtime/date.cc)
//   runtime::Vector::Sort                             (runtime/vector.cc:45-110)
#include <cstdint>

#include "runtime/date.h"
#include "runtime/vector.h"

extern "C" {

int32_t kdbref_build_date(int32_t y, int32_t m, int32_t d) {
  return static_cast<int32_t>(kush::runtime::Date::DateBuilder(y, m, d).Build());
}

void kdbref_split_date(int32_t jd, int32_t* y, int32_t* m, int32_t* d) {
  kush::runtime::Date::SplitDate(jd, y, m, d);
}

// Sorts (key, payload) int32 pairs with the reference merge sort and a strict
// less-than on the key (the ORDER BY comparator shape), so the tie order of
// the reference can be compared with the oracle's.
static bool LessKey(int8_t* a, int8_t* b) {
  return *reinterpret_cast<int32_t*>(a) < *reinterpret_cast<int32_t*>(b);
}

void kdbref_sort_pairs(int32_t* pairs, int32_t n) {
  kush::runtime::Vector::Vector v;
  kush::runtime::Vector::Create(&v, 8, n > 0 ? n : 1);
  for (int32_t i = 0; i < n; i++) {
    auto* slot = reinterpret_cast<int32_t*>(kush::runtime::Vector::PushBack(&v));
    slot[0] = pairs[2 * i];
    slot[1] = pairs[2 * i + 1];
  }
  kush::runtime::Vector::Sort(&v, &LessKey);
  for (int32_t i = 0; i < n; i++) {
    auto* slot = reinterpret_cast<int32_t*>(kush::runtime::Vector::Get(&v, i));
    pairs[2 * i] = slot[0];
    pairs[2 * i + 1] = slot[1];
  }
  kush::runtime::Vector::Free(&v);
}

}  // extern "C"
