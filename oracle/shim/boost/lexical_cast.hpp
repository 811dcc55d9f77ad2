// Build shim: decimal text of a 128-bit integer, the only lexical_cast use
// of the reference (Types.hpp:30-36).
#pragma once
#include <string>
namespace boost {
template <class To, class From>
To lexical_cast(From v) {
    const bool neg = v < 0;
    unsigned __int128 u = neg ? (unsigned __int128)0 - (unsigned __int128)v : (unsigned __int128)v;
    std::string s;
    do {
        s.insert(s.begin(), char('0' + int(u % 10)));
        u /= 10;
    } while (u != 0);
    if (neg) s.insert(s.begin(), '-');
    return s;
}
}  // namespace boost
