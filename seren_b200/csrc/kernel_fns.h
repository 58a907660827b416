// kernel_fns.h - the kernel functions of setup/kernel.F90 (M4 and M4
// Thomas-Couchman, NDIM = 3, GRAD_H_SPH) at the centre of table bin i,
// s = (2i+1)/KERNTOT (kernel.F90:58).
//
// One definition serves the host tables (tables.cpp) and device code that
// evaluates a bin instead of loading it.  Expressions keep the Fortran
// association; gfortran expands x**n for constant integer n into the
// multiplication chains below; the host side is compiled without FMA
// contraction and the device side with -fmad=false, and the expressions use
// only +, -, * and /, which IEEE rounds the same way on both, so a value
// computed on the device equals the table entry bit for bit.
#pragma once

#if defined(__CUDACC__)
#define SEREN_HD __host__ __device__ __forceinline__
#else
#define SEREN_HD inline
#endif

namespace seren {
namespace kfn {

constexpr int KERNTOT = 10000;
constexpr int KERN1 = 5000;                        // int(HALFKERNTOT)
constexpr double INVPI = 0.318309886;
constexpr double NDIMPR = 3.0;

SEREN_HD double pw2(double x) { return x * x; }
SEREN_HD double pw3(double x) { return x * (x * x); }
SEREN_HD double pw4(double x) { const double x2 = x * x; return x2 * x2; }
SEREN_HD double pw5(double x) { const double x2 = x * x; const double x3 = x * x2; return x2 * x3; }

// bin centre (KERNRANGE*i + 1) * (1/KERNTOT)
SEREN_HD double bin_s(int i) { return (2.0 * (double)i + 1.0) * (1.0 / (double)KERNTOT); }

// the Thomas-Couchman boundary int(KERNTOT/3)
SEREN_HD int kern_tc() { return (int)((double)KERNTOT / 3.0); }

SEREN_HD double w0(int i) {
  const double s = bin_s(i);
  if (i < KERN1) return ((1.0 - (1.5 * s) * s) + 0.75 * pw3(s)) * INVPI;
  return (0.25 * pw3(2.0 - s)) * INVPI;
}

SEREN_HD double w4(int i) {
  const double s = bin_s(i);
  if (i < KERN1) return (-(3.0 * s) + (2.25 * s) * s) * INVPI;
  const double saux = 2.0 - s;
  return (-((0.75 * saux) * saux)) * INVPI;
}

SEREN_HD double w1(int i, int kernel) {
  const double s = bin_s(i);
  if (i < KERN1) {
    const double a1 = (kernel == 1 && i < kern_tc()) ? -1.0 : -(3.0 * s) + (2.25 * s) * s;
    return a1 * INVPI;
  }
  const double saux = 2.0 - s;
  return (-((0.75 * saux) * saux)) * INVPI;
}

SEREN_HD double w5(int i) {
  const double s = bin_s(i);
  if (i < KERN1) return ((4.0 / 3.0) * s - 1.2 * pw3(s)) + 0.5 * pw4(s);
  return ((((8.0 / 3.0) * s - 3.0 * pw2(s)) + 1.2 * pw3(s)) - (1.0 / 6.0) * pw4(s)) -
         1.0 / (15.0 * pw2(s));
}

SEREN_HD double w6(int i) {
  const double s = bin_s(i);
  if (i < KERN1) return ((7.0 / 5.0 - (2.0 / 3.0) * pw2(s)) + 0.3 * pw4(s)) - 0.1 * pw5(s);
  return (((((-(1.0 / (15.0 * s))) + 8.0 / 5.0) - (4.0 / 3.0) * pw2(s)) + pw3(s)) - 0.3 * pw4(s)) +
         (1.0 / 30.0) * pw5(s);
}

SEREN_HD double wh(int i) {
  const double s = bin_s(i);
  if (i < KERN1)
    return ((-NDIMPR + ((1.5 * (NDIMPR + 2.0)) * s) * s) - (0.75 * (NDIMPR + 3.0)) * pw3(s)) * INVPI;
  return (((-2.0 * NDIMPR + (3.0 * (NDIMPR + 1.0)) * s) - ((1.50 * (NDIMPR + 2.0)) * s) * s) +
          (0.25 * (NDIMPR + 3.0)) * pw3(s)) * INVPI;
}

SEREN_HD double wg(int i) {
  const double s = bin_s(i);
  if (i < KERN1) return ((1.4 - (2.0 * s) * s) + 1.5 * pw4(s)) - 0.6 * pw5(s);
  return (((1.6 - (4.0 * s) * s) + 4.0 * pw3(s)) - 1.5 * pw4(s)) + 0.2 * pw5(s);
}

}  // namespace kfn
}  // namespace seren
