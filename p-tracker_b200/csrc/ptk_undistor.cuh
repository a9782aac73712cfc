// undistor of the reference (src/distortion_correction.cpp:20-61: Brown
// radial K1-K3 and tangential P1-P3 about (xc, yc), then a two-axis parallax
// scaling) on the device.  The cos/sin of the two parallax angles come from
// the host; files including this header are compiled with -fmad=false so the
// FP64 operations are the CPU's, one for one.
#pragma once

#include <cmath>

namespace ptk {

struct Disto {
  double p[14];
  double trig[4];  // cos t1, -sin t1, -sin t2, cos t2
};

inline Disto make_disto(const double* params14) {
  Disto d;
  for (int k = 0; k < 14; ++k) d.p[k] = params14[k];
  d.trig[0] = std::cos(params14[10]);
  d.trig[1] = -std::sin(params14[10]);
  d.trig[2] = -std::sin(params14[12]);
  d.trig[3] = std::cos(params14[12]);
  return d;
}

__device__ __forceinline__ void undistor_d(const Disto& X, double xd, double yd, double* xo, double* yo) {
  const double Xc = X.p[0], Yc = X.p[1], K1 = X.p[2], K2 = X.p[3], K3 = X.p[4];
  const double P1 = X.p[5], P2 = X.p[6], P3 = X.p[7];
  const double dx = xd - Xc;
  const double dy = yd - Yc;
  const double r2 = dx * dx + dy * dy;
  const double r4 = r2 * r2;
  const double r6 = r4 * r2;
  const double xu = xd + dx * (K1 * r2 + K2 * r4 + K3 * r6) + (P1 * (r2 + 2.0 * dx * dx) + 2.0 * P2 * dx * dy) * (1.0 + P3 * r2);
  const double yu = yd + dy * (K1 * r2 + K2 * r4 + K3 * r6) + (2.0 * P1 * dx * dy + P2 * (r2 + 2.0 * dy * dy)) * (1.0 + P3 * r2);
  const double Xcp = X.p[8], Ycp = X.p[9], parallax1 = X.p[11], parallax2 = X.p[13];
  const double nx1 = X.trig[0], ny1 = X.trig[1], nx2 = X.trig[2], ny2 = X.trig[3];
  const double dX = xu - Xcp;
  const double dY = yu - Ycp;
  const double S1 = (1.0 + parallax1) * (dX * nx1 + dY * ny1);
  const double S2 = (1.0 + parallax2) * (dX * nx2 + dY * ny2);
  *xo = Xcp + S1 * nx1 + S2 * nx2;
  *yo = Ycp + S1 * ny1 + S2 * ny2;
}

}  // namespace ptk
