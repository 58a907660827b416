// tables.cpp - the kernel tables of setup/kernel.F90 (M4 and M4 Thomas-Couchman,
// NDIM = 3, GRAD_H_SPH), built on the host once per context and uploaded.
//
// Entry i holds the kernel functions at the bin centre s = (2i+1)/KERNTOT
// (kernel.F90:58), evaluated by the shared definitions of kernel_fns.h; this
// file is compiled without FMA contraction, so the values equal those of the
// reference's own tables.
#include <vector>

#include "kernel_fns.h"

namespace seren {

void make_kernel_tables(int kernel, std::vector<double>& w0, std::vector<double>& w1,
                        std::vector<double>& w4, std::vector<double>& w5, std::vector<double>& w6,
                        std::vector<double>& wh, std::vector<double>& wg) {
  const int n = kfn::KERNTOT + 1;
  w0.assign(n, 0.0); w1.assign(n, 0.0); w4.assign(n, 0.0); w5.assign(n, 0.0);
  w6.assign(n, 0.0); wh.assign(n, 0.0); wg.assign(n, 0.0);
  for (int i = 0; i < n; ++i) {
    w0[i] = kfn::w0(i);
    w1[i] = kfn::w1(i, kernel);
    w4[i] = kfn::w4(i);
    wh[i] = kfn::wh(i);
    w5[i] = kfn::w5(i);
    w6[i] = kfn::w6(i);
    wg[i] = kfn::wg(i);
  }
}

}  // namespace seren
