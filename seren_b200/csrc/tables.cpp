// tables.cpp - the kernel tables of setup/kernel.F90 (M4 and M4 Thomas-Couchman,
// NDIM = 3, GRAD_H_SPH), built on the host once per context and uploaded.
//
// Entry i holds the kernel functions at the bin centre s = (2i+1)/KERNTOT
// (kernel.F90:58).  Expressions keep the Fortran association; gfortran expands
// x**n for constant integer n into the multiplication chain used below, and
// this file is compiled without FMA contraction, so the values equal those of
// the reference's own tables.
#include <vector>

namespace seren {

namespace {
inline double pw2(double x) { return x * x; }
inline double pw3(double x) { return x * (x * x); }
inline double pw4(double x) { const double x2 = x * x; return x2 * x2; }
inline double pw5(double x) { const double x2 = x * x; const double x3 = x * x2; return x2 * x3; }
}  // namespace

void make_kernel_tables(int kernel, std::vector<double>& w0, std::vector<double>& w1,
                        std::vector<double>& w4, std::vector<double>& w5, std::vector<double>& w6,
                        std::vector<double>& wh, std::vector<double>& wg) {
  constexpr int KERNTOT = 10000;
  constexpr double KERNRANGE = 2.0, NDIMPR = 3.0, INVPI = 0.318309886;
  const int n = KERNTOT + 1;
  w0.assign(n, 0.0); w1.assign(n, 0.0); w4.assign(n, 0.0); w5.assign(n, 0.0);
  w6.assign(n, 0.0); wh.assign(n, 0.0); wg.assign(n, 0.0);
  const double invkerntot = 1.0 / (double)KERNTOT;
  const int kern1 = 5000;                          // int(HALFKERNTOT)
  const int kerntc = (int)((double)KERNTOT / 3.0); // Thomas-Couchman boundary
  for (int i = 0; i <= KERNTOT; ++i) {
    const double s = (KERNRANGE * (double)i + 1.0) * invkerntot;
    const double saux = KERNRANGE - s;
    double a0, a1, a4, a5, a6, ah, ag;
    if (i < kern1) {
      a1 = (kernel == 1 && i < kerntc) ? -1.0 : -(3.0 * s) + (2.25 * s) * s;
      a0 = (1.0 - (1.5 * s) * s) + 0.75 * pw3(s);
      a4 = -(3.0 * s) + (2.25 * s) * s;
      a5 = ((4.0 / 3.0) * s - 1.2 * pw3(s)) + 0.5 * pw4(s);
      a6 = ((7.0 / 5.0 - (2.0 / 3.0) * pw2(s)) + 0.3 * pw4(s)) - 0.1 * pw5(s);
      ah = (-NDIMPR + ((1.5 * (NDIMPR + 2.0)) * s) * s) - (0.75 * (NDIMPR + 3.0)) * pw3(s);
      ag = ((1.4 - (2.0 * s) * s) + 1.5 * pw4(s)) - 0.6 * pw5(s);
    } else {
      a0 = 0.25 * pw3(saux);
      a1 = -((0.75 * saux) * saux);
      a4 = -((0.75 * saux) * saux);
      a5 = ((((8.0 / 3.0) * s - 3.0 * pw2(s)) + 1.2 * pw3(s)) - (1.0 / 6.0) * pw4(s)) -
           1.0 / (15.0 * pw2(s));
      a6 = (((((-(1.0 / (15.0 * s))) + 8.0 / 5.0) - (4.0 / 3.0) * pw2(s)) + pw3(s)) - 0.3 * pw4(s)) +
           (1.0 / 30.0) * pw5(s);
      ah = ((-2.0 * NDIMPR + (3.0 * (NDIMPR + 1.0)) * s) - ((1.50 * (NDIMPR + 2.0)) * s) * s) +
           (0.25 * (NDIMPR + 3.0)) * pw3(s);
      ag = (((1.6 - (4.0 * s) * s) + 4.0 * pw3(s)) - 1.5 * pw4(s)) + 0.2 * pw5(s);
    }
    w0[i] = a0 * INVPI;
    w1[i] = a1 * INVPI;
    w4[i] = a4 * INVPI;
    wh[i] = ah * INVPI;
    w5[i] = a5;
    w6[i] = a6;
    wg[i] = ag;
  }
}

}  // namespace seren
