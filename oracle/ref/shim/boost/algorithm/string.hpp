// Test-only stand-in for the one Boost facility the reference's gas-optics class uses
// (boost::trim, src_cuda/Gas_optics_rrtmgp.cu:113): strip leading and trailing blanks.
#pragma once
#include <string>

namespace boost {
inline void trim(std::string& s)
{
    const char* ws = " \t\n\r\f\v";
    const size_t a = s.find_first_not_of(ws);
    if (a == std::string::npos) { s.clear(); return; }
    const size_t b = s.find_last_not_of(ws);
    s = s.substr(a, b - a + 1);
}
}  // namespace boost
