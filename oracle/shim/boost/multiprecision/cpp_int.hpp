// Build shim for compiling the reference's Math.hpp / Sieve.hpp without Boost.
// The reference uses boost::multiprecision::int128_t / uint128_t only as
// 128-bit integers (Types.hpp:11-12); every hot-path value is below 2^63 in
// magnitude, where the compiler's __int128 gives the same results.
#pragma once
namespace boost {
namespace multiprecision {
using int128_t = __int128;
using uint128_t = unsigned __int128;
}  // namespace multiprecision
}  // namespace boost
