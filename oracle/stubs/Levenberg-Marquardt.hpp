// ORACLE / TEST INFRASTRUCTURE ONLY.
// Declaration-level stand-in for toofus' Levenberg-Marquardt.hpp (included at
// src/p-tracker.hpp:50).  It is used only by the distortion-parameter fit
// (src/distortion_correction.cpp:409-475), which is outside the tracking path;
// lmdif1 here reports "not available" and leaves x unchanged.
#pragma once
#include <string>
namespace levmar {
inline int get_lwa(int m, int n) { return m * n + 5 * n + m; }
template <class FCN>
inline int lmdif1(FCN, void*, int, int, double*, double*, double, int*, double*, int) { return 0; }
inline std::string getInfo(int) { return "levmar stub: not available in the oracle build"; }
}  // namespace levmar
