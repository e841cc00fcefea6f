// Compiled CPU baseline loops -- TEST / BENCHMARK INFRASTRUCTURE ONLY.
//
// Filled in below: hand-restated versions of the scalar loops the reference's
// translators generate for the benchmark plans, timed single-threaded as the
// CPU reference arm.
#include <cstdint>
