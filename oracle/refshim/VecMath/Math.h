// Shim (oracle test infrastructure): VecMath fast functions mapped to std::.
#pragma once
#include <cmath>
namespace vecMath {
template <class R> R FastExp(R x) { return std::exp(x); }
template <class R> R FastLog(R x) { return std::log(x); }
template <class R> R FastSin(R x) { return std::sin(x); }
template <class R> R FastCos(R x) { return std::cos(x); }
template <class R> void FastSinCos(R x, R &s, R &c) { s = std::sin(x); c = std::cos(x); }
template <class R> R FastPow(R x, R n) { return std::pow(x, n); }
template <class R> R IntPow(R x, int n) { return std::pow(x, n); }
} // namespace vecMath
