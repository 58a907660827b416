// seren_oracle.cpp - TEST INFRASTRUCTURE ONLY (the checker, never the product).
//
// CPU FP64 restatement of the SEREN grad-h SPH force hot path.  Each routine
// follows the Fortran file cited beside it statement by statement, with the
// same left-to-right association of every expression and no FMA contraction
// (built with -ffp-contract=off, as gfortran -O3 on x86-64 emits no FMA).
// Fortran x**n with an integer constant n is expanded the way gfortran does it
// (the powi multiplication chain); x**y with a real exponent calls libm pow.
//
// Parity status: UNPINNED.  The reference has no golden vectors or fixtures
// for this path and cannot be compiled here (no Fortran compiler); see
// seren_oracle.h.  Particle ids inside this file are 0-based; the C ABI
// converts with params.index_base.
#include "seren_oracle.h"

#include <omp.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

namespace {

// headers/macros.h constants (NDIM=3, M4 kernel, double precision PR)
constexpr int KERNTOT = 10000;                // macros.h:102
constexpr double HALFKERNTOT = 5000.0;        // macros.h:103
constexpr double KERNRANGE = 2.0;             // macros.h:105
constexpr double KERNRANGESQD = 4.0;          // macros.h:106
constexpr double INVKERNRANGE = 0.5;          // macros.h:107
constexpr double INVPI = 0.318309886;         // macros.h:14
constexpr double ONETHIRD = 0.333333333;      // macros.h:18 (INVNDIM, :49)
constexpr double NDIMPR = 3.0;                // macros.h:47
constexpr double NDIMPLUS1 = 4.0;             // macros.h:50
constexpr double SMALL_NUMBER = 1.0e-20;      // macros.h:84
constexpr double BIG_NUMBER = 9.9e20;         // macros.h:82
constexpr double HMULT = 1.1;                 // macros.h:98
constexpr double H_CON = 0.02;                // macros.h:171
constexpr int GRADH_ITERATION_MAX = 20;       // macros.h:172
constexpr int LEAFMAX = 8;                    // macros.h:138
constexpr int LISTSIZE = 10000;               // macros.h:189
constexpr int GLISTSIZE = 10000;              // macros.h:190
constexpr int HGROW_CAP = 2000;               // guard: the reference loops forever if ptot < pp_gather

// gfortran's expansion of x**n for integer constant n (powi chain)
inline double pw2(double x) { return x * x; }
inline double pw3(double x) { return x * (x * x); }
inline double pw4(double x) { double x2 = x * x; return x2 * x2; }
inline double pw5(double x) { double x2 = x * x; double x3 = x * x2; return x2 * x3; }
inline double pw6(double x) { double x3 = x * (x * x); return x3 * x3; }

struct Tables {
  std::vector<double> w0, w1, w2, w3, w4, w5, w6, wh, wg;
};

// setup/kernel.F90:14-266, M4 (and M4TC) kernel, NDIM=3, GRAD_H_SPH
void make_tables(int kernel, Tables& t) {
  const int n = KERNTOT + 1;
  t.w0.assign(n, 0); t.w1.assign(n, 0); t.w2.assign(n, 0); t.w3.assign(n, 0);
  t.w4.assign(n, 0); t.w5.assign(n, 0); t.w6.assign(n, 0); t.wh.assign(n, 0); t.wg.assign(n, 0);
  const double invkerntot = 1.0 / (double)KERNTOT;           // kernel.F90:40
  const int kern1 = (int)HALFKERNTOT;                        // :42
  const int kerntc = (int)((double)KERNTOT / 3.0);           // :44
  for (int i = 0; i <= KERNTOT; ++i) {
    const double s = (KERNRANGE * (double)i + 1.0) * invkerntot;  // :58
    const double saux = KERNRANGE - s;                             // :59
    double w0, w1, w2, w3, w4, w5, w6, wh, wg;
    if (i < kern1) {                                                // :63
      if (kernel == 1 && i < kerntc) w1 = -1.0;                     // :66-70
      else w1 = -(3.0 * s) + (2.25 * s) * s;                        // :73
      w0 = (1.0 - (1.5 * s) * s) + 0.75 * pw3(s);                   // :75
      w2 = ((4.0 / 3.0) * pw3(s) - 1.2 * pw5(s)) + 0.5 * pw6(s);    // :76
      w3 = (((7.0 / 5.0) * s - (2.0 / 3.0) * pw3(s)) + 0.3 * pw5(s)) - 0.1 * pw6(s);  // :77-78
      w4 = -(3.0 * s) + (2.25 * s) * s;                             // :79
      w5 = ((4.0 / 3.0) * s - 1.2 * pw3(s)) + 0.5 * pw4(s);         // :80
      w6 = ((7.0 / 5.0 - (2.0 / 3.0) * pw2(s)) + 0.3 * pw4(s)) - 0.1 * pw5(s);  // :81-82
      wh = (-NDIMPR + ((1.5 * (NDIMPR + 2.0)) * s) * s) - (0.75 * (NDIMPR + 3.0)) * pw3(s);  // :86-87
      wg = ((1.4 - (2.0 * s) * s) + 1.5 * pw4(s)) - 0.6 * pw5(s);   // :88
    } else {
      w0 = 0.25 * pw3(saux);                                        // :92
      w1 = -((0.75 * saux) * saux);                                 // :93
      w2 = ((((8.0 / 3.0) * pw3(s) - 3.0 * pw4(s)) + 1.2 * pw5(s)) - (1.0 / 6.0) * pw6(s)) - (1.0 / 15.0);  // :94-95
      w3 = (((((-(1.0 / 15.0)) + (8.0 / 5.0) * s) - (4.0 / 3.0) * pw3(s)) + pw4(s)) - 0.3 * pw5(s)) +
           (1.0 / 30.0) * pw6(s);                                   // :96-97
      w4 = -((0.75 * saux) * saux);                                 // :98
      w5 = ((((8.0 / 3.0) * s - 3.0 * pw2(s)) + 1.2 * pw3(s)) - (1.0 / 6.0) * pw4(s)) -
           1.0 / (15.0 * pw2(s));                                   // :99-100
      w6 = (((((-(1.0 / (15.0 * s))) + 8.0 / 5.0) - (4.0 / 3.0) * pw2(s)) + pw3(s)) - 0.3 * pw4(s)) +
           (1.0 / 30.0) * pw5(s);                                   // :101-102
      wh = ((-2.0 * NDIMPR + (3.0 * (NDIMPR + 1.0)) * s) - ((1.50 * (NDIMPR + 2.0)) * s) * s) +
           (0.25 * (NDIMPR + 3.0)) * pw3(s);                        // :105-106
      wg = (((1.6 - (4.0 * s) * s) + 4.0 * pw3(s)) - 1.5 * pw4(s)) + 0.2 * pw5(s);  // :107
    }
    // 3-D normalisation, kernel.F90:120-125
    w0 = w0 * INVPI; w1 = w1 * INVPI; w4 = w4 * INVPI; wh = wh * INVPI;
    t.w0[i] = w0; t.w1[i] = w1; t.w2[i] = w2; t.w3[i] = w3; t.w4[i] = w4;
    t.w5[i] = w5; t.w6[i] = w6; t.wh[i] = wh; t.wg[i] = wg;
  }
}

// headers/modules.F90:907-959 node types (plist holds 0-based particle ids)
struct GravNode {
  int leaf = 0, nextcell = 0, ifopen = -1;
  int plist[LEAFMAX];
  double r[3], m, dminsqd, q[5];
};
struct HydroNode {
  int leaf = 0, nextcell = 0, ifopen = -1;
  int plist[LEAFMAX];
  double r[3], rmax, hrangemax;
};
struct StockNode {
  double hmax, bbmin[3], bbmax[3];
};
struct TempNode {
  int childof[8];
  int pfirst, plast, leaf, nextcell, ifopen;
  int plist[LEAFMAX];
  double r[3];
};

using clk = std::chrono::steady_clock;
inline double secs(clk::time_point a, clk::time_point b) {
  return std::chrono::duration<double>(b - a).count();
}

}  // namespace

struct seren_oracle {
  seren_gpu_params prm{};
  int64_t pmax = 0;
  int ptot = 0;
  Tables tab;
  std::vector<double> parray;  // [p*6 + k]: x, y, z, m, h, zeta
  std::vector<double> v;       // [p*3 + k]
  std::vector<double> rho, omega, div_v, drhodt, press, sound;
  std::vector<int> pptot, pplist;  // pplist[p*pp_limit + k]
  int cmax = 0, ctot = -1, ltot = 0;
  std::vector<int> first_cell, last_cell;
  std::vector<GravNode> grav;
  std::vector<HydroNode> hyd;
  std::vector<StockNode> stock;
  std::vector<TempNode> temp;
  double rextent = 0.0;
  bool have_tree = false;
  seren_oracle_counts cnt{};
  double stage[6] = {0, 0, 0, 0, 0, 0};
  std::string err;

  int fail(int code, const std::string& msg) {
    err = msg;
    return code;
  }
  int base() const { return prm.index_base; }

  // ------------------------------------------------------------------------
  // main/bounding_box.F90:9-43
  void bounding_box(double rmax[3], double rmin[3]) {
    for (int k = 0; k < 3; ++k) { rmax[k] = -BIG_NUMBER; rmin[k] = BIG_NUMBER; }
    for (int p = 0; p < ptot; ++p)
      for (int k = 0; k < 3; ++k) {
        rmax[k] = std::max(rmax[k], parray[p * 6 + k]);
        rmin[k] = std::min(rmin[k], parray[p * 6 + k]);
      }
    rextent = std::max(std::max(rmax[0] - rmin[0], rmax[1] - rmin[1]), rmax[2] - rmin[2]);
  }

  // BHtree/BHgrav_build.F90:12-309 (linked-list octree, serial child numbering)
  int build() {
    std::vector<int> cellof(ptot), nextptcl(ptot), whichchild(ptot);
    for (int p = 0; p < ptot; ++p) { cellof[p] = 0; nextptcl[p] = p + 1; }   // :46-49
    temp.assign(cmax + 1, TempNode());
    grav.assign(cmax + 1, GravNode());
    for (int c = 0; c <= cmax; ++c) {                                        // :51-56
      for (int k = 0; k < 8; ++k) temp[c].childof[k] = -2;
      temp[c].pfirst = -1; temp[c].plast = -1; temp[c].leaf = 0;
      temp[c].ifopen = -1; temp[c].nextcell = cmax + 1;
      for (int k = 0; k < LEAFMAX; ++k) temp[c].plist[k] = -1;
      grav[c].ifopen = -1;
      for (int k = 0; k < LEAFMAX; ++k) grav[c].plist[k] = -1;
    }
    temp[0].pfirst = 0; temp[0].plast = ptot - 1;                            // :58-59
    first_cell.assign(prm.lmax + 1, 0); last_cell.assign(prm.lmax + 1, 0);   // :60-61
    double rmax[3], rmin[3];
    bounding_box(rmax, rmin);                                                // :65
    double cellsize = 0.5 * std::max(std::max(rmax[0] - rmin[0], rmax[1] - rmin[1]), rmax[2] - rmin[2]);
    for (int k = 0; k < 3; ++k) temp[0].r[k] = 0.5 * (rmin[k] + rmax[k]);    // :67
    int l = 0;
    ctot = 0;
    temp[0].leaf = 0;
    temp[0].nextcell = cmax + 1;                                             // :75
    grav[0].leaf = 0; grav[0].nextcell = cmax + 1;
    std::vector<int> templist{0};
    while (true) {
      cellsize = 0.5 * cellsize;                                             // :95
      const int nlist = (int)templist.size();
      // :107-142 octant of every particle of every cell on this level
#pragma omp parallel for schedule(guided, 1)
      for (int j = 0; j < nlist; ++j) {
        const int c = templist[j];
        int p = temp[c].pfirst;
        const double rc0 = temp[c].r[0], rc1 = temp[c].r[1], rc2 = temp[c].r[2];
        while (true) {
          int ckid = 1;
          if (parray[p * 6 + 0] > rc0) ckid += 1;
          if (parray[p * 6 + 1] > rc1) ckid += 2;
          if (parray[p * 6 + 2] > rc2) ckid += 4;
          whichchild[p] = ckid;
          temp[c].childof[ckid - 1] = -1;
          if (p == temp[c].plast) break;
          p = nextptcl[p];
        }
      }
      // :149-157 serial numbering of the new children
      for (int j = 0; j < nlist; ++j) {
        const int c = templist[j];
        for (int k = 0; k < 8; ++k)
          if (temp[c].childof[k] == -1) {
            ctot = ctot + 1;
            if (ctot > cmax) return fail(SEREN_GPU_ERR_CAPACITY, "cell count exceeds cmax = 2*ptot");
            temp[c].childof[k] = ctot;
          }
      }
      // :165-255 distribute particles, make leaves, child centres and links
#pragma omp parallel for schedule(guided, 1) if (l > 0)
      for (int j = 0; j < nlist; ++j) {
        const int c = templist[j];
        int nptclin[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        int p = temp[c].pfirst;
        while (true) {
          const int ckid = temp[c].childof[whichchild[p] - 1];
          cellof[p] = ckid;
          if (temp[ckid].pfirst == -1) temp[ckid].pfirst = p;
          else nextptcl[temp[ckid].plast] = p;
          temp[ckid].plast = p;
          nptclin[whichchild[p] - 1] += 1;
          if (p == temp[c].plast) break;
          p = nextptcl[p];
        }
        int nkids = 0;
        int clist[8];
        const double rc[3] = {temp[c].r[0], temp[c].r[1], temp[c].r[2]};
        for (int k = 1; k <= 8; ++k) {
          if (nptclin[k - 1] == 0) continue;
          const int ckid = temp[c].childof[k - 1];
          if (nptclin[k - 1] > 0 && nptclin[k - 1] <= LEAFMAX) {
            temp[ckid].leaf = nptclin[k - 1];
            int i = 0;
            int pp = temp[ckid].pfirst;
            while (true) {
              temp[ckid].plist[i++] = pp;
              if (pp == temp[ckid].plast) break;
              pp = nextptcl[pp];
            }
          } else if (nptclin[k - 1] > LEAFMAX) {
            temp[ckid].leaf = 0;
          }
          if (k == 1 || k == 3 || k == 5 || k == 7) temp[ckid].r[0] = rc[0] - cellsize;   // :212-216
          else temp[ckid].r[0] = rc[0] + cellsize;
          if (k == 1 || k == 2 || k == 5 || k == 6) temp[ckid].r[1] = rc[1] - cellsize;   // :218-222
          else temp[ckid].r[1] = rc[1] + cellsize;
          if (k < 5) temp[ckid].r[2] = rc[2] - cellsize;                                 // :224-228
          else temp[ckid].r[2] = rc[2] + cellsize;
          clist[nkids++] = ckid;
        }
        temp[c].ifopen = clist[0];                                            // :239
        for (int k = 0; k < nkids - 1; ++k) temp[clist[k]].nextcell = clist[k + 1];
        temp[clist[nkids - 1]].nextcell = temp[c].nextcell;
        grav[c].ifopen = temp[c].ifopen;
        for (int k = 0; k < nkids; ++k) {
          const int ckid = clist[k];
          grav[ckid].leaf = temp[ckid].leaf;
          grav[ckid].nextcell = temp[ckid].nextcell;
          grav[ckid].ifopen = temp[ckid].leaf > 0 ? -1 : temp[ckid].ifopen;
          for (int i = 0; i < LEAFMAX; ++i) grav[ckid].plist[i] = temp[ckid].plist[i];
        }
      }
      l = l + 1;                                                              // :260-262
      first_cell[l] = last_cell[l - 1] + 1;
      last_cell[l] = ctot;
      templist.clear();                                                       // :270-278
      bool alldone = true;
      for (int c = first_cell[l]; c <= last_cell[l]; ++c)
        if (temp[c].leaf == 0) { alldone = false; templist.push_back(c); }
      if (alldone) break;
      if (l >= prm.lmax) return fail(SEREN_GPU_ERR_LMAX, "Reached maximum level");   // :289
    }
    ltot = l;
    // leaves have no first child; the reference leaves ifopen unset for them
    for (int c = 0; c <= ctot; ++c) if (grav[c].leaf > 0) grav[c].ifopen = -1;
    have_tree = true;
    return SEREN_GPU_OK;
  }

  // BHtree/BH_reorder_particles.F90:57-78 + main/reorder_array.F90
  void reorder(std::vector<int>& dummylist) {
    dummylist.resize(ptot);
    for (int p = 0; p < ptot; ++p) dummylist[p] = p;
    int gascount = 0;
    int c = 0;
    while (true) {
      if (grav[c].leaf > 0) {
        for (int i = 0; i < grav[c].leaf; ++i) {
          const int p = grav[c].plist[i];
          dummylist[gascount] = p;
          grav[c].plist[i] = gascount;
          gascount++;
        }
        c = grav[c].nextcell;
      } else if (grav[c].leaf == 0) {
        c = grav[c].ifopen;
      } else {
        c = grav[c].nextcell;
      }
      if (c > ctot) break;
    }
    std::vector<double> np(parray.size()), nv(v.size());
    for (int i = 0; i < ptot; ++i) {
      const int p = dummylist[i];
      for (int k = 0; k < 6; ++k) np[i * 6 + k] = parray[p * 6 + k];
      if (!v.empty()) for (int k = 0; k < 3; ++k) nv[i * 3 + k] = v[p * 3 + k];
    }
    parray.swap(np);
    if (!v.empty()) v.swap(nv);
    auto perm1 = [&](std::vector<double>& a) {
      if (a.empty()) return;
      std::vector<double> b(a.size());
      for (int i = 0; i < ptot; ++i) b[i] = a[dummylist[i]];
      a.swap(b);
    };
    perm1(rho); perm1(omega); perm1(div_v); perm1(drhodt); perm1(press); perm1(sound);
  }

  // BHtree/BHgrav_stock.F90:11-358 (QUADRUPOLE, GEOMETRIC_MAC)
  void grav_stock() {
    stock.assign(ctot + 1, StockNode());
    for (int c = 0; c <= ctot; ++c) {                                         // :43-48
      grav[c].dminsqd = 0.0;
      stock[c].hmax = 0.0;
      for (int k = 0; k < 3; ++k) { stock[c].bbmin[k] = BIG_NUMBER; stock[c].bbmax[k] = -BIG_NUMBER; }
    }
    const double daux = 10.0 * std::pow(1.7976931348623157e308, -0.2);       // :347
    for (int l = ltot; l >= 0; --l) {
#pragma omp parallel for if (l > 1)
      for (int c = first_cell[l]; c <= last_cell[l]; ++c) {
        GravNode& g = grav[c];
        StockNode& s = stock[c];
        double mc = 0.0;
        int nalive = 0;
        double rc[3] = {0.0, 0.0, 0.0};
        double dr[3];
        if (g.leaf == -1) {                                                   // :80-96
          for (int k = 0; k < 3; ++k) g.r[k] = 0.0;
          g.m = 0.0;
          for (int k = 0; k < 5; ++k) g.q[k] = 0.0;
          s.hmax = 0.0;
          for (int k = 0; k < 3; ++k) { s.bbmin[k] = -0.0; s.bbmax[k] = 0.0; }
          g.dminsqd = 0.0;
          continue;
        } else if (g.leaf == 1) {                                             // :100-113
          const int p = g.plist[0];
          for (int k = 0; k < 3; ++k) rc[k] = parray[p * 6 + k];
          for (int k = 0; k < 3; ++k) g.r[k] = rc[k];
          g.m = parray[p * 6 + 3];
          for (int k = 0; k < 5; ++k) g.q[k] = 0.0;
          s.hmax = parray[p * 6 + 4];
          for (int k = 0; k < 3; ++k) { s.bbmin[k] = rc[k]; s.bbmax[k] = rc[k]; }
        } else if (g.leaf > 0) {                                              // :118-183
          const int npart = g.leaf;
          for (int i = 0; i < npart; ++i) {
            const int p = g.plist[i];
            const double mp = parray[p * 6 + 3];
            mc = mc + mp;
            s.hmax = std::max(s.hmax, parray[p * 6 + 4]);
            for (int k = 0; k < 3; ++k) rc[k] = rc[k] + mp * parray[p * 6 + k];
            for (int k = 0; k < 3; ++k) {
              s.bbmax[k] = std::max(s.bbmax[k], parray[p * 6 + k]);
              s.bbmin[k] = std::min(s.bbmin[k], parray[p * 6 + k]);
            }
          }
          for (int k = 0; k < 3; ++k) rc[k] = rc[k] / mc;
          double qc[5] = {0, 0, 0, 0, 0};
          for (int i = 0; i < npart; ++i) {
            const int p = g.plist[i];
            for (int k = 0; k < 3; ++k) dr[k] = parray[p * 6 + k] - rc[k];
            const double mp = parray[p * 6 + 3];
            const double drsqd = (dr[0] * dr[0] + dr[1] * dr[1]) + dr[2] * dr[2];
            qc[0] = qc[0] + mp * ((3.0 * dr[0]) * dr[0] - drsqd);
            qc[1] = qc[1] + mp * ((3.0 * dr[0]) * dr[1]);
            qc[2] = qc[2] + mp * ((3.0 * dr[1]) * dr[1] - drsqd);
            qc[3] = qc[3] + mp * ((3.0 * dr[2]) * dr[0]);
            qc[4] = qc[4] + mp * ((3.0 * dr[2]) * dr[1]);
          }
          g.m = mc;
          for (int k = 0; k < 3; ++k) g.r[k] = rc[k];
          for (int k = 0; k < 5; ++k) g.q[k] = qc[k];
        } else {                                                              // :188-312
          const int cfirst = g.ifopen;
          const int cend = g.nextcell;
          int cc = cfirst;
          while (true) {
            if (grav[cc].leaf >= 0) {
              nalive = nalive + 1;
              mc = mc + grav[cc].m;
              for (int k = 0; k < 3; ++k) rc[k] = rc[k] + grav[cc].m * grav[cc].r[k];
              s.hmax = std::max(stock[cc].hmax, s.hmax);
              for (int k = 0; k < 3; ++k) {
                s.bbmax[k] = std::max(stock[cc].bbmax[k], s.bbmax[k]);
                s.bbmin[k] = std::min(stock[cc].bbmin[k], s.bbmin[k]);
              }
            }
            cc = grav[cc].nextcell;
            if (cc == cend) break;
          }
          if (nalive == 0) {                                                  // :213-227
            g.leaf = -1;
            for (int k = 0; k < 3; ++k) g.r[k] = BIG_NUMBER;
            g.m = 0.0;
            for (int k = 0; k < 5; ++k) g.q[k] = 0.0;
            s.hmax = BIG_NUMBER;
            for (int k = 0; k < 3; ++k) { s.bbmin[k] = -BIG_NUMBER; s.bbmax[k] = BIG_NUMBER; }
            continue;
          }
          if (mc > 0.0) for (int k = 0; k < 3; ++k) rc[k] = rc[k] / mc;       // :230
          double qc[5] = {0, 0, 0, 0, 0};
          cc = cfirst;
          while (true) {
            if (grav[cc].leaf == -1) {                                        // :240-244 (quirk kept)
              cc = g.nextcell;
              if (cc == cend) break;
              continue;
            }
            const double mcc = grav[cc].m;
            for (int k = 0; k < 5; ++k) qc[k] = qc[k] + grav[cc].q[k];
            for (int k = 0; k < 3; ++k) dr[k] = grav[cc].r[k] - rc[k];
            const double drsqd = (dr[0] * dr[0] + dr[1] * dr[1]) + dr[2] * dr[2];
            qc[0] = qc[0] + mcc * ((3.0 * dr[0]) * dr[0] - drsqd);
            qc[1] = qc[1] + mcc * ((3.0 * dr[0]) * dr[1]);
            qc[2] = qc[2] + mcc * ((3.0 * dr[1]) * dr[1] - drsqd);
            qc[3] = qc[3] + mcc * ((3.0 * dr[2]) * dr[0]);
            qc[4] = qc[4] + mcc * ((3.0 * dr[2]) * dr[1]);
            cc = grav[cc].nextcell;
            if (cc == cend) break;
          }
          g.m = mc;
          for (int k = 0; k < 3; ++k) g.r[k] = rc[k];
          for (int k = 0; k < 5; ++k) g.q[k] = qc[k];
        }
        // :317-348 MAC quantities
        for (int k = 0; k < 3; ++k) dr[k] = std::max(s.bbmax[k] - rc[k], rc[k] - s.bbmin[k]);
        const double diagonalsqd = (dr[0] * dr[0] + dr[1] * dr[1]) + dr[2] * dr[2];
        const double rsize = std::sqrt(diagonalsqd) + KERNRANGE * s.hmax;
        if (prm.thetamaxsqd > 0.0) g.dminsqd = diagonalsqd / prm.thetamaxsqd;
        else g.dminsqd = BIG_NUMBER;
        g.dminsqd = std::max(g.dminsqd, rsize * rsize);
        if (g.dminsqd < daux) g.dminsqd = daux;
      }
    }
  }

  // BHtree/copy_BHgrav_to_BHhydro.F90:11-37
  void copy_to_hydro() {
    hyd.assign(ctot + 1, HydroNode());
    for (int c = 0; c <= ctot; ++c) {
      hyd[c].leaf = grav[c].leaf;
      hyd[c].nextcell = grav[c].nextcell;
      hyd[c].ifopen = grav[c].ifopen;
      for (int k = 0; k < LEAFMAX; ++k) hyd[c].plist[k] = grav[c].plist[k];
      hyd[c].hrangemax = 0.0;
    }
  }

  // BHtree/BHhydro_stock.F90:10-174
  void hydro_stock() {
    for (int c = 0; c <= ctot; ++c)
      for (int k = 0; k < 3; ++k) { stock[c].bbmin[k] = BIG_NUMBER; stock[c].bbmax[k] = -BIG_NUMBER; }
    for (int l = ltot; l >= 0; --l) {
#pragma omp parallel for if (l > 2)
      for (int c = first_cell[l]; c <= last_cell[l]; ++c) {
        HydroNode& h = hyd[c];
        StockNode& s = stock[c];
        int nalive = 0;
        double rc[3], halfbox[3];
        if (h.leaf == -1) {
          for (int k = 0; k < 3; ++k) h.r[k] = 0.0;
          h.rmax = 0.0; h.hrangemax = 0.0;
          for (int k = 0; k < 3; ++k) { s.bbmin[k] = 0.0; s.bbmax[k] = 0.0; }
        } else if (h.leaf == 1) {
          const int p = h.plist[0];
          for (int k = 0; k < 3; ++k) rc[k] = parray[p * 6 + k];
          for (int k = 0; k < 3; ++k) h.r[k] = rc[k];
          h.rmax = 0.0;
          for (int k = 0; k < 3; ++k) { s.bbmin[k] = rc[k]; s.bbmax[k] = rc[k]; }
        } else if (h.leaf > 0) {
          for (int i = 0; i < h.leaf; ++i) {
            const int p = h.plist[i];
            for (int k = 0; k < 3; ++k) {
              s.bbmax[k] = std::max(s.bbmax[k], parray[p * 6 + k]);
              s.bbmin[k] = std::min(s.bbmin[k], parray[p * 6 + k]);
            }
          }
          double diagonalsqd = 0.0;
          for (int k = 0; k < 3; ++k) {
            rc[k] = 0.5 * (s.bbmax[k] + s.bbmin[k]);
            halfbox[k] = s.bbmax[k] - rc[k];
            diagonalsqd = diagonalsqd + halfbox[k] * halfbox[k];
          }
          for (int k = 0; k < 3; ++k) h.r[k] = rc[k];
          h.rmax = std::sqrt(diagonalsqd);
        } else {
          int cc = h.ifopen;
          const int cend = h.nextcell;
          while (true) {
            if (hyd[cc].leaf >= 0) {
              nalive = nalive + 1;
              for (int k = 0; k < 3; ++k) {
                s.bbmax[k] = std::max(stock[cc].bbmax[k], s.bbmax[k]);
                s.bbmin[k] = std::min(stock[cc].bbmin[k], s.bbmin[k]);
              }
            }
            cc = hyd[cc].nextcell;
            if (cc == cend) break;
          }
          if (nalive == 0) {
            h.leaf = -1;
            for (int k = 0; k < 3; ++k) h.r[k] = BIG_NUMBER;
            h.rmax = 0.0; h.hrangemax = 0.0;
            for (int k = 0; k < 3; ++k) { s.bbmin[k] = BIG_NUMBER; s.bbmax[k] = BIG_NUMBER; }
            continue;
          }
          double diagonalsqd = 0.0;
          for (int k = 0; k < 3; ++k) {
            rc[k] = 0.5 * (s.bbmax[k] + s.bbmin[k]);
            halfbox[k] = s.bbmax[k] - rc[k];
            diagonalsqd = diagonalsqd + halfbox[k] * halfbox[k];
          }
          for (int k = 0; k < 3; ++k) h.r[k] = rc[k];
          h.rmax = std::sqrt(diagonalsqd);
        }
      }
    }
  }

  // BHtree/BHhydro_update_hmax.F90:29-88
  void update_hmax() {
    for (int l = ltot; l >= 0; --l) {
#pragma omp parallel for if (l > 2)
      for (int c = first_cell[l]; c <= last_cell[l]; ++c) {
        HydroNode& h = hyd[c];
        double hrangemax = 0.0;
        if (h.leaf == -1) {
          h.hrangemax = 0.0;
        } else if (h.leaf == 1) {
          h.hrangemax = KERNRANGE * parray[h.plist[0] * 6 + 4];
        } else if (h.leaf > 0) {
          for (int i = 0; i < h.leaf; ++i)
            hrangemax = std::max(hrangemax, KERNRANGE * parray[h.plist[i] * 6 + 4]);
          h.hrangemax = hrangemax;
        } else {
          int cc = h.ifopen;
          const int cend = h.nextcell;
          while (true) {
            hrangemax = std::max(hrangemax, hyd[cc].hrangemax);
            cc = hyd[cc].nextcell;
            if (cc == cend) break;
          }
          h.hrangemax = hrangemax;
        }
      }
    }
  }

  // BHtree/BHhydro_hguess.F90:11-163 (GRAD_H_SPH: number criterion)
  void hguess() {
    std::vector<int> levelof(ctot + 1, 0), pcontained(ctot + 1, 0);
    for (int l = ltot; l >= 0; --l) {
      for (int c = first_cell[l]; c <= last_cell[l]; ++c) {
        levelof[c] = l;
        if (hyd[c].leaf > 0) {
          pcontained[c] = hyd[c].leaf;
        } else if (hyd[c].leaf == 0) {
          int cc = hyd[c].ifopen;
          const int cend = hyd[c].nextcell;
          while (true) {
            pcontained[c] = pcontained[c] + pcontained[cc];
            cc = hyd[cc].nextcell;
            if (cc == cend) break;
          }
        }
      }
    }
    std::vector<int> pstack(prm.lmax + 1, 0);
    std::vector<double> rstack(prm.lmax + 1, 0.0);
    const int thresh = (int)(0.5 * (double)prm.pp_gather);
    int c = 0;
    while (true) {
      const int l = levelof[c];
      pstack[l] = pcontained[c];
      rstack[l] = hyd[c].rmax;
      if (hyd[c].leaf > 0) {
        int laux = l;
        while (true) {
          if (pstack[laux] > thresh || laux == 0) break;
          laux = laux - 1;
        }
        const double hg = INVKERNRANGE * rstack[laux];
        for (int i = 0; i < hyd[c].leaf; ++i) parray[hyd[c].plist[i] * 6 + 4] = hg;
        c = hyd[c].nextcell;
      } else if (hyd[c].leaf == 0) {
        c = hyd[c].ifopen;
      } else {
        c = hyd[c].nextcell;
      }
      if (c > ctot) break;
    }
  }

  // BHtree/BHhydrowalk_hgather.F90:11-77 (gather-only candidate walk)
  int hgather_walk(const double rp[3], double hrange, int pp_max, std::vector<int>& list,
                   int64_t& nodes) const {
    int c = 0;
    int pp_pot = 0;
    list.clear();
    while (true) {
      ++nodes;
      const HydroNode& h = hyd[c];
      const double d0 = h.r[0] - rp[0], d1 = h.r[1] - rp[1], d2 = h.r[2] - rp[2];
      const double drsqd = (d0 * d0 + d1 * d1) + d2 * d2;
      const double t = hrange + h.rmax;
      const double maxdistsqd = t * t;
      if (drsqd <= maxdistsqd) {
        if (h.leaf > 0) {
          if (pp_pot + h.leaf > pp_max) return -1;
          for (int i = 0; i < h.leaf; ++i) { list.push_back(h.plist[i]); pp_pot++; }
          c = h.nextcell;
        } else if (h.leaf == 0) {
          c = h.ifopen;
        } else {
          c = h.nextcell;
        }
      } else {
        c = h.nextcell;
      }
      if (c > cmax) break;
    }
    return pp_pot;
  }

  // sph/h_gather.F90:14-203 (BH_TREE, insertion sort, no MINIMUM_H): h from
  // exactly pp_gather neighbours.  distance2 is main/distance2.F90:30-60
  // (dr = r_pp - r_p, dr1^2 + dr2^2 + dr3^2 left to right).  The reference
  // loops forever when fewer than pp_gather other particles exist; here the
  // search stops once h_high passes 1e6 root extents (SEREN_GPU_ERR_WALK).
  int h_gather(int p, double& hguess, int64_t& nodes) const {
    const double rp[3] = {parray[p * 6 + 0], parray[p * 6 + 1], parray[p * 6 + 2]};
    const int pp_gather = prm.pp_gather;
    int pp_pot = 0;                                                       // :46-55
    int pp_max = LISTSIZE;
    const double h_old = hguess;
    double h_high = HMULT * h_old;
    double h_low = h_old / HMULT;
    double h_search = 0.0;
    double hrangesqd_high = (KERNRANGESQD * h_high) * h_high;
    std::vector<int> potlist;
    std::vector<int> high_list(pp_max);
    std::vector<double> rsqd_high(pp_max);
    int pp_low = 0, pp_high = 0;
    const double hcap = 1.0e6 * (rextent > 0.0 ? rextent : 1.0);
    while (true) {                                                        // :62-160
      while (true) {                                                      // :66-107
        if (h_high > h_search) {
          h_search = HMULT * h_high;
          pp_pot = hgather_walk(rp, KERNRANGE * h_search, pp_max, potlist, nodes);
        }
        if (pp_pot < 0) {                                                 // :92-101
          h_search = 0.0;
          pp_pot = 0;
          pp_max = ptot;
          high_list.assign(pp_max, 0);
          rsqd_high.assign(pp_max, 0.0);
        } else if (pp_pot <= pp_gather) {                                 // :102-107
          pp_pot = 0;
          h_search = 0.0;
          h_low = h_high;
          h_high = HMULT * h_high;
          hrangesqd_high = (KERNRANGESQD * h_high) * h_high;
          if (h_high > hcap) return SEREN_GPU_ERR_WALK;
        }
        if (pp_pot > 0) break;
      }
      int pp_tot = 0;                                                     // :111-113
      pp_high = 0;
      pp_low = 0;
      hrangesqd_high = (KERNRANGESQD * h_high) * h_high;
      const double hrangesqd_low = (KERNRANGESQD * h_low) * h_low;
      for (int i = 0; i < pp_pot; ++i) {                                  // :120-139
        const int pp = potlist[i];
        if (pp == p) continue;
        const double dr0 = parray[pp * 6 + 0] - rp[0];
        const double dr1 = parray[pp * 6 + 1] - rp[1];
        const double dr2 = parray[pp * 6 + 2] - rp[2];
        const double drsqd = (dr0 * dr0 + dr1 * dr1) + dr2 * dr2;
        if (drsqd < hrangesqd_high) {
          if (drsqd < hrangesqd_low) {
            pp_low = pp_low + 1;
          } else {
            pp_high = pp_high + 1;
            high_list[pp_high - 1] = pp;
            rsqd_high[pp_high - 1] = drsqd;
          }
        }
        if (pp_high == pp_max) break;
      }
      pp_tot = pp_low + pp_high;                                          // :143
      if (pp_tot < pp_gather) {                                           // :147-151
        h_low = h_high;
        h_high = HMULT * h_high;
        hrangesqd_high = (KERNRANGESQD * h_high) * h_high;
        if (h_high > hcap) return SEREN_GPU_ERR_WALK;
        continue;
      } else if (pp_low >= pp_gather) {                                   // :154-157
        h_high = h_low;
        h_low = h_low / HMULT;
        continue;
      } else {                                                            // :160-162
        break;
      }
    }
    // insertion sort of the annulus (sorts/insertion_sort.F90), then the
    // (pp_gather - pp_low)-th smallest, :179-183
    for (int j = 1; j < pp_high; ++j) {
      const double a = rsqd_high[j];
      const int ia = high_list[j];
      int i = j - 1;
      while (i >= 0 && rsqd_high[i] > a) {
        rsqd_high[i + 1] = rsqd_high[i];
        high_list[i + 1] = high_list[i];
        --i;
      }
      rsqd_high[i + 1] = a;
      high_list[i + 1] = ia;
    }
    const double drsqd = rsqd_high[pp_gather - pp_low - 1];
    hguess = INVKERNRANGE * std::sqrt(drsqd);
    return SEREN_GPU_OK;
  }

  // BHtree/BHhydro_walk.F90:9-80 (gather and scatter candidate walk)
  int hydro_walk(const double rp[3], double hrange, int pp_max, std::vector<int>& list) const {
    int c = 0;
    int pp_pot = 0;
    list.clear();
    while (true) {
      const HydroNode& h = hyd[c];
      const double d0 = h.r[0] - rp[0], d1 = h.r[1] - rp[1], d2 = h.r[2] - rp[2];
      const double drsqd = (d0 * d0 + d1 * d1) + d2 * d2;
      const double t1 = hrange + h.rmax;
      const double t2 = h.hrangemax + h.rmax;
      if (drsqd <= t1 * t1 || drsqd <= t2 * t2) {
        if (h.leaf > 0) {
          if (pp_pot + h.leaf > pp_max) return -1;
          for (int i = 0; i < h.leaf; ++i) { list.push_back(h.plist[i]); pp_pot++; }
          c = h.nextcell;
        } else if (h.leaf == 0) {
          c = h.ifopen;
        } else {
          c = h.nextcell;
        }
      } else {
        c = h.nextcell;
      }
      if (c > cmax) break;
    }
    return pp_pot;
  }

  // sph/all_sph_gradh.F90:11-492 (GRAD_H_SPH, BH_TREE, GRAVITY, no MHD)
  int all_sph_gradh(int p, std::vector<int>& potlist, seren_oracle_counts& lc) {
    const double* w0 = tab.w0.data();
    const double* wh = tab.wh.data();
    const double* w4 = tab.w4.data();
    const double* wg = tab.wg.data();
    const double h_fac = prm.h_fac;
    const double rp[3] = {parray[p * 6 + 0], parray[p * 6 + 1], parray[p * 6 + 2]};
    const double mp = parray[p * 6 + 3];
    double hp = parray[p * 6 + 4];
    const double vp[3] = {v[p * 3 + 0], v[p * 3 + 1], v[p * 3 + 2]};
    double rhotemp = rho[p];
    double omega_p = omega[p];
    double div_v_p;
    double invhp = 1.0 / hp;                                             // :132
    double hfactor_p = std::pow(invhp, NDIMPR);                          // :133
    double hrangesqd = (KERNRANGESQD * hp) * hp;                         // :134
    int iteration = 0;
    const double h_old = hp;
    double h_new = hp;
    double h_high = 0.0;
    double h_upper = rextent;
    double h_lower = 0.0;
    int pp_pot = 0;
    int pp_max = std::min(LISTSIZE, ptot);
    int ngrow = 0;
    while (true) {
      while (true) {                                                      // :154-191
        if (hp > h_high) {
          pp_pot = 0;
          h_high = hp * HMULT;
          pp_pot = hgather_walk(rp, KERNRANGE * h_high, pp_max, potlist, lc.grav_nodes);
          lc.gradh_walks++;
        }
        if (pp_pot < 0) {
          h_high = 0.0;
          pp_pot = 0;
          pp_max = ptot;
        } else if (pp_pot < prm.pp_gather) {
          h_high = 0.0;
          pp_pot = 0;
          hp = hp * HMULT;
          if (++ngrow > HGROW_CAP) return fail(SEREN_GPU_ERR_WALK, "grad-h: fewer particles than pp_gather");
        }
        if (pp_pot > 0) break;
      }
      h_new = hp;                                                          // :199-202
      invhp = 1.0 / hp;
      hfactor_p = std::pow(invhp, NDIMPR);
      hrangesqd = (KERNRANGESQD * hp) * hp;
      rhotemp = (mp * w0[0]) * hfactor_p;                                  // :209
      omega_p = ((mp * hfactor_p) * invhp) * wh[0];                        // :210
      for (int i = 0; i < pp_pot; ++i) {                                   // :214-235
        const int pp = potlist[i];
        if (pp == p) continue;
        lc.gradh_tests++;
        const double d0 = parray[pp * 6 + 0] - rp[0];
        const double d1 = parray[pp * 6 + 1] - rp[1];
        const double d2 = parray[pp * 6 + 2] - rp[2];
        const double drsqd = (d0 * d0 + d1 * d1) + d2 * d2;
        if (drsqd >= hrangesqd) continue;
        const double drmag = std::sqrt(drsqd) + SMALL_NUMBER;
        const double skern = (HALFKERNTOT * drmag) * invhp;
        const int kern = (int)skern;
        if (kern >= KERNTOT) continue;
        lc.gradh_pairs++;
        const double mpp = parray[pp * 6 + 3];
        rhotemp = rhotemp + (mpp * hfactor_p) * w0[kern];
        omega_p = omega_p + ((mpp * hfactor_p) * invhp) * wh[kern];
      }
      lc.gradh_passes++;
      omega_p = 1.0 + ((hp * omega_p) / (NDIMPR * rhotemp));              // :238
      if (std::fabs(hp - h_fac * std::pow(mp / rhotemp, ONETHIRD)) / hp < H_CON &&
          iteration >= 1)
        break;                                                             // :246-247
      if (iteration < GRADH_ITERATION_MAX) {                               // :252-281
        h_new = h_fac * std::pow(mp / rhotemp, ONETHIRD);
      } else if (iteration == GRADH_ITERATION_MAX) {
        lc.gradh_bisections++;
        h_upper = rextent;
        h_lower = 0.0;
        h_new = 0.5 * (h_lower + h_upper);
      } else if (iteration < 2 * GRADH_ITERATION_MAX) {
        double fbisection;
        if (rhotemp > SMALL_NUMBER)
          fbisection = std::pow(hp, NDIMPR) - (std::pow(h_fac, NDIMPR) * mp) / rhotemp;
        else
          fbisection = 1.0;
        if (fbisection > 0.0) h_upper = hp;
        else h_lower = hp;
        h_new = 0.5 * (h_lower + h_upper);
      } else {
        h_new = h_old;
        hp = h_new;
        break;
      }
      hp = h_new;                                                          // :284-285
      iteration = iteration + 1;
    }
    hp = h_fac * std::pow(mp / rhotemp, ONETHIRD);                         // :317
    invhp = 1.0 / hp;
    hfactor_p = std::pow(invhp, NDIMPR);
    hrangesqd = (KERNRANGESQD * hp) * hp;
    rhotemp = (mp * w0[0]) * hfactor_p;                                    // :323
    omega_p = ((mp * hfactor_p) * invhp) * wh[0];
    div_v_p = 0.0;
    double zeta_p = ((mp * invhp) * invhp) * wg[0];                        // :346
    for (int i = 0; i < pp_pot; ++i) {                                     // :360-425
      const int pp = potlist[i];
      if (pp == p) continue;
      lc.gradh_final_tests++;
      const double d0 = parray[pp * 6 + 0] - rp[0];
      const double d1 = parray[pp * 6 + 1] - rp[1];
      const double d2 = parray[pp * 6 + 2] - rp[2];
      double drmag = (d0 * d0 + d1 * d1) + d2 * d2;
      if (drmag > hrangesqd) continue;
      drmag = std::sqrt(drmag) + SMALL_NUMBER;
      const double skern = (HALFKERNTOT * drmag) * invhp;
      const int kern = (int)skern;
      if (kern > KERNTOT) continue;
      lc.gradh_final_pairs++;
      const double mpp = parray[pp * 6 + 3];
      const double dv0 = v[pp * 3 + 0] - vp[0];
      const double dv1 = v[pp * 3 + 1] - vp[1];
      const double dv2 = v[pp * 3 + 2] - vp[2];
      const double dvdr = (dv0 * d0 + dv1 * d1) + dv2 * d2;
      rhotemp = rhotemp + (mpp * hfactor_p) * w0[kern];
      omega_p = omega_p + ((mpp * hfactor_p) * invhp) * wh[kern];
      div_v_p = div_v_p - ((((mpp * dvdr) * w4[kern]) * hfactor_p) * invhp) / drmag;
      zeta_p = zeta_p + ((mpp * invhp) * invhp) * wg[kern];
    }
    omega_p = 1.0 + ((hp * omega_p) / (NDIMPR * rhotemp));                // :428
    div_v_p = div_v_p / rhotemp;
    rho[p] = rhotemp;                                                      // :436-442
    omega[p] = omega_p;
    div_v[p] = div_v_p;
    drhodt[p] = -((rhotemp * div_v_p) / omega_p);
    parray[p * 6 + 4] = hp;
    parray[p * 6 + 5] = -((hp * zeta_p) / ((NDIMPR * rhotemp) * omega_p));
    if (parray[p * 6 + 4] < 0.0) return fail(SEREN_GPU_ERR_NEGATIVE_H, "Negative smoothing lengths");
    return SEREN_GPU_OK;
  }

  // sph/get_neib.F90:10-140 (and get_neib_on_fly.F90:11-130 with list capture)
  int neib_list(int p, double hp, std::vector<int>& pot, std::vector<int>& out,
                int64_t& tests) const {
    const double rp[3] = {parray[p * 6 + 0], parray[p * 6 + 1], parray[p * 6 + 2]};
    const double hrangesqd_p = (KERNRANGESQD * hp) * hp;
    int pp_max = std::min(LISTSIZE, ptot);
    int pp_pot;
    while (true) {
      pp_pot = hydro_walk(rp, KERNRANGE * hp, pp_max, pot);
      if (pp_pot < 0) pp_max = ptot;
      else break;
    }
    out.clear();
    int pp_tot = 0;
    for (int i = 0; i < pp_pot; ++i) {
      const int pp = pot[i];
      if (pp == p) continue;
      tests++;
      const double hpp = parray[pp * 6 + 4];
      const double hrangesqd_pp = (KERNRANGESQD * hpp) * hpp;
      const double d0 = parray[pp * 6 + 0] - rp[0];
      const double d1 = parray[pp * 6 + 1] - rp[1];
      const double d2 = parray[pp * 6 + 2] - rp[2];
      const double drsqd = (d0 * d0 + d1 * d1) + d2 * d2;
      if (drsqd <= hrangesqd_p || drsqd <= hrangesqd_pp) {
        pp_tot++;
        out.push_back(pp);
      }
    }
    return pp_tot;
  }

  void get_neib_all(const std::vector<int>& act, seren_oracle_counts& c) {
    const int L = prm.pp_limit;
    int64_t tests = 0, pairs = 0;
#pragma omp parallel reduction(+ : tests, pairs)
    {
      std::vector<int> pot, out;
#pragma omp for schedule(dynamic, 64)
      for (int i = 0; i < (int)act.size(); ++i) {
        const int p = act[i];
        const int pp_tot = neib_list(p, parray[p * 6 + 4], pot, out, tests);
        pptot[p] = pp_tot;
        pairs += pp_tot;
        if (pp_tot <= L)
          for (int k = 0; k < pp_tot; ++k) pplist[(size_t)p * L + k] = out[k];
      }
    }
    c.neib_tests += tests;
    c.neib_pairs += pairs;
  }

  // sph/hydro_gradh.F90:9-339 (NEIGHBOUR_LISTS, MON97, no TD/Balsara)
  void hydro_gradh(int p, std::vector<int>& pot, std::vector<int>& lst, double out[3],
                   int64_t& npair, int64_t& nvisc) const {
    const double* w1 = tab.w1.data();
    const double rp[3] = {parray[p * 6 + 0], parray[p * 6 + 1], parray[p * 6 + 2]};
    const double hp = parray[p * 6 + 4];
    const double invhp = 1.0 / hp;
    const double hfactor_p = std::pow(invhp, NDIMPLUS1);
    const double vp[3] = {v[p * 3 + 0], v[p * 3 + 1], v[p * 3 + 2]};
    const double sound_p = sound[p];
    const double rho_p = rho[p];
    const double pfactor_p = ((press[p] / rho_p) / rho_p) / omega[p];
    double at[3] = {0, 0, 0}, ad[3] = {0, 0, 0};
    const int L = prm.pp_limit;
    int pp_numb = pptot[p];
    const int* list;
    if (pp_numb <= L) {
      list = &pplist[(size_t)p * L];
    } else {
      int64_t dummy = 0;
      pp_numb = neib_list(p, hp, pot, lst, dummy);
      list = lst.data();
    }
    const double alpha = prm.alpha;
    for (int i = 0; i < pp_numb; ++i) {
      const int pp = list[i];
      double wmean = 0.0;
      const double rho_pp = rho[pp];
      const double mpp = parray[pp * 6 + 3];
      const double hpp = parray[pp * 6 + 4];
      double du[3] = {parray[pp * 6 + 0] - rp[0], parray[pp * 6 + 1] - rp[1], parray[pp * 6 + 2] - rp[2]};
      double drmag = (du[0] * du[0] + du[1] * du[1]) + du[2] * du[2];
      if (drmag >= (KERNRANGESQD * hp) * hp && drmag >= (KERNRANGESQD * hpp) * hpp) continue;
      npair++;
      drmag = std::sqrt(drmag) + SMALL_NUMBER;
      const double dv0 = v[pp * 3 + 0] - vp[0];
      const double dv1 = v[pp * 3 + 1] - vp[1];
      const double dv2 = v[pp * 3 + 2] - vp[2];
      const double dvdr = (dv0 * du[0] + dv1 * du[1]) + dv2 * du[2];
      const double invdrmag = 1.0 / drmag;
      for (int k = 0; k < 3; ++k) du[k] = du[k] * invdrmag;
      const double pfactor_pp = ((press[pp] / rho_pp) / rho_pp) / omega[pp];
      if (drmag < KERNRANGE * hp) {
        const double skern = (HALFKERNTOT * drmag) * invhp;
        int kern = (int)skern;
        kern = std::min(kern, KERNTOT);
        wmean = (0.5 * hfactor_p) * w1[kern];
        for (int k = 0; k < 3; ++k) at[k] = at[k] + (((mpp * pfactor_p) * hfactor_p) * w1[kern]) * du[k];
      }
      if (drmag < KERNRANGE * hpp) {
        const double invhpp = 1.0 / hpp;
        const double hfactor_pp = std::pow(invhpp, NDIMPLUS1);
        const double skern = (HALFKERNTOT * drmag) * invhpp;
        int kern = (int)skern;
        kern = std::min(kern, KERNTOT);
        wmean = wmean + (0.5 * hfactor_pp) * w1[kern];
        for (int k = 0; k < 3; ++k) at[k] = at[k] + (((mpp * pfactor_pp) * hfactor_pp) * w1[kern]) * du[k];
      }
      const double rhomean = 0.5 * (rho_p + rho_pp);
      if (dvdr < 0.0) {
        nvisc++;
        const double beta = 2.0 * alpha;
        const double alpha_mean = alpha;
        const double vsignal = (sound_p + sound[pp]) - ((beta * dvdr) * invdrmag);
        for (int k = 0; k < 3; ++k)
          ad[k] = ad[k] - ((((((mpp * alpha_mean) * vsignal) * dvdr) * invdrmag) * du[k]) * wmean) / rhomean;
      }
    }
    for (int k = 0; k < 3; ++k) out[k] = at[k] + ad[k];
  }

  // gravity/gravity_gradh.F90:11-95
  inline void gravity_gradh(double invhp, double hpp, double mpp, const double rp[3],
                            const double rpp[3], double zo_p, double zo_pp, double at[3],
                            double& dpotp) const {
    const double* w4 = tab.w4.data();
    const double* w5 = tab.w5.data();
    const double* w6 = tab.w6.data();
    const double dr[3] = {rpp[0] - rp[0], rpp[1] - rp[1], rpp[2] - rp[2]};
    const double drsqd = (dr[0] * dr[0] + dr[1] * dr[1]) + dr[2] * dr[2];
    const double drmag = std::sqrt(drsqd) + SMALL_NUMBER;
    const double invdrmag = 1.0 / drmag;
    double grav;
    if (invdrmag > INVKERNRANGE * invhp) {
      int kern = (int)((HALFKERNTOT * drmag) * invhp);
      kern = std::min(kern, KERNTOT);
      grav = (invhp * invhp) * (w5[kern] + ((zo_p * w4[kern]) * invhp) * invhp);
      dpotp = invhp * w6[kern];
    } else {
      grav = invdrmag * invdrmag;
      dpotp = invdrmag;
    }
    if (drmag < KERNRANGE * hpp) {
      const double invhpp = 1.0 / hpp;
      int kern = (int)((HALFKERNTOT * drmag) * invhpp);
      kern = std::min(kern, KERNTOT);
      grav = grav + (invhpp * invhpp) * (w5[kern] + ((zo_pp * w4[kern]) * invhpp) * invhpp);
      dpotp = dpotp + invhpp * w6[kern];
    } else {
      grav = grav + invdrmag * invdrmag;
      dpotp = dpotp + invdrmag;
    }
    for (int k = 0; k < 3; ++k) at[k] = (((0.5 * mpp) * invdrmag) * grav) * dr[k];
    dpotp = (0.5 * mpp) * dpotp;
  }

  // gravity/gravity_meanh.F90:12-69
  inline void gravity_meanh(double hmean, double mpp, const double rp[3], const double rpp[3],
                            double at[3], double& dpotp) const {
    const double* w5 = tab.w5.data();
    const double* w6 = tab.w6.data();
    const double dr[3] = {rpp[0] - rp[0], rpp[1] - rp[1], rpp[2] - rp[2]};
    const double drsqd = (dr[0] * dr[0] + dr[1] * dr[1]) + dr[2] * dr[2];
    const double drmag = std::sqrt(drsqd) + SMALL_NUMBER;
    const double invdrmag = 1.0 / drmag;
    double grav;
    if (drmag < KERNRANGE * hmean) {
      const double invhmean = 1.0 / hmean;
      int kern = (int)((HALFKERNTOT * drmag) * invhmean);
      kern = std::min(kern, KERNTOT);
      grav = ((invdrmag * invhmean) * invhmean) * w5[kern];
      dpotp = invhmean * w6[kern];
    } else {
      grav = pw3(invdrmag);
      dpotp = invdrmag;
    }
    for (int k = 0; k < 3; ++k) at[k] = (mpp * grav) * dr[k];
    dpotp = mpp * dpotp;
  }

  // BHtree/BHgrav_accel.F90:21-348 (GEOMETRIC_MAC, QUADRUPOLE, GRAD_H_SPH);
  // pself >= 0: SPH particle pself; pself < 0: a sink with smoothing length
  // 1/invhp (near field by gravity_meanh, :299-314).
  void bhgrav_accel(int pself, double invhp, const double rp[3], double agravp[3], double& potp,
                    std::vector<int>& treelist, int64_t& ncell, int64_t& npair,
                    int64_t& nnode) const {
    agravp[0] = agravp[1] = agravp[2] = 0.0;
    potp = 0.0;
    int nlist = 0;
    const double zo_p = pself < 0 ? 0.0 : parray[pself * 6 + 5];
    const double hp = 1.0 / invhp;
    treelist.resize(GLISTSIZE);
    int c = 0;
    while (true) {
      ++nnode;
      const GravNode& g = grav[c];
      if (g.leaf == 1) {                                                     // :128-136
        const int pp = g.plist[0];
        if (pp != pself) treelist[nlist++] = pp;
        c = g.nextcell;
      } else {
        const double dr[3] = {rp[0] - g.r[0], rp[1] - g.r[1], rp[2] - g.r[2]};   // :146-147
        const double drsqd = (dr[0] * dr[0] + dr[1] * dr[1]) + dr[2] * dr[2];
        if (drsqd > g.dminsqd) {                                                 // :155
          ++ncell;
          const double invdrsqd = 1.0 / (drsqd + SMALL_NUMBER);
          const double invdrmag = std::sqrt(invdrsqd);
          double at[3];
          for (int k = 0; k < 3; ++k) at[k] = -(((g.m * invdrsqd) * invdrmag) * dr[k]);
          double dpot = g.m * invdrmag;
          const double invdr5 = (invdrsqd * invdrsqd) * invdrmag;
          const double* q = g.q;
          const double qscalar = (((q[0] * dr[0]) * dr[0] + (q[2] * dr[1]) * dr[1]) -
                                  ((q[0] + q[2]) * dr[2]) * dr[2]) +
                                 2.0 * ((((q[1] * dr[0]) * dr[1]) + ((q[3] * dr[0]) * dr[2])) +
                                        ((q[4] * dr[1]) * dr[2]));
          at[0] = (at[0] + (((q[0] * dr[0] + q[1] * dr[1]) + q[3] * dr[2]) * invdr5)) -
                  ((((2.5 * qscalar) * dr[0]) * invdr5) * invdrsqd);
          at[1] = (at[1] + (((q[1] * dr[0] + q[2] * dr[1]) + q[4] * dr[2]) * invdr5)) -
                  ((((2.5 * qscalar) * dr[1]) * invdr5) * invdrsqd);
          at[2] = (at[2] + (((q[3] * dr[0] + q[4] * dr[1]) - (q[0] + q[2]) * dr[2]) * invdr5)) -
                  ((((2.5 * qscalar) * dr[2]) * invdr5) * invdrsqd);
          dpot = dpot + (0.5 * qscalar) * invdr5;
          for (int k = 0; k < 3; ++k) agravp[k] = agravp[k] + at[k];
          potp = potp + dpot;
          c = g.nextcell;
        } else {
          if (g.leaf > 0) {                                                  // :242-253
            for (int i = 0; i < g.leaf; ++i) {
              const int pp = g.plist[i];
              if (pp == pself) continue;
              treelist[nlist++] = pp;
            }
            c = g.nextcell;
          } else if (g.leaf == 0) {
            c = g.ifopen;
          } else {
            c = g.nextcell;
          }
        }
      }
      if (nlist > GLISTSIZE - LEAFMAX || (nlist > 0 && c > ctot)) {        // :272-314
        for (int i = 0; i < nlist; ++i) {
          const int pp = treelist[i];
          const double* rpp = &parray[pp * 6];
          double at[3], dpot;
          if (pself >= 0)
            gravity_gradh(invhp, rpp[4], rpp[3], rp, rpp, zo_p, rpp[5], at, dpot);
          else
            gravity_meanh(0.5 * (hp + rpp[4]), rpp[3], rp, rpp, at, dpot);
          for (int k = 0; k < 3; ++k) agravp[k] = agravp[k] + at[k];
          potp = potp + dpot;
        }
        npair += nlist;
        nlist = 0;
      }
      if (c > ctot) break;
    }
  }

  // sinks/direct_sink_gravity.F90:10-64 (s_self < 0: a gas particle)
  void direct_sink_gravity(int s_self, double hp, const double rp[3], int nsink,
                           const double* sink, double agravp[3], double& potp) const {
    agravp[0] = agravp[1] = agravp[2] = 0.0;
    potp = 0.0;
    for (int ss = 0; ss < nsink; ++ss) {
      if (ss == s_self) continue;
      const double* sr = &sink[ss * 5];
      double at[3], dpot;
      gravity_meanh(0.5 * (hp + sr[4]), sr[3], rp, sr, at, dpot);
      for (int k = 0; k < 3; ++k) agravp[k] = agravp[k] + at[k];
      potp = potp + dpot;
    }
  }

  std::vector<int> active_list(const int32_t* acclist, int32_t nacc) const {
    std::vector<int> act;
    if (acclist == nullptr) {
      act.resize(ptot);
      for (int p = 0; p < ptot; ++p) act[p] = p;
    } else {
      act.resize(nacc);
      for (int i = 0; i < nacc; ++i) act[i] = acclist[i] - base();
    }
    return act;
  }
  bool active_ok(const std::vector<int>& act) const {
    for (int p : act) if (p < 0 || p >= ptot) return false;
    return true;
  }
};

extern "C" {

int seren_oracle_set_threads(int32_t nthreads) {
  if (nthreads > 0) omp_set_num_threads(nthreads);
  return omp_get_max_threads();
}

int seren_oracle_kernel_tables(int32_t kernel, double* out) {
  Tables t;
  make_tables(kernel, t);
  const std::vector<double>* ws[9] = {&t.w0, &t.w1, &t.w2, &t.w3, &t.w4, &t.w5, &t.w6, &t.wh, &t.wg};
  for (int j = 0; j < 9; ++j) std::memcpy(out + (size_t)j * (KERNTOT + 1), ws[j]->data(), sizeof(double) * (KERNTOT + 1));
  return SEREN_GPU_OK;
}

int seren_oracle_create(seren_oracle** out, int64_t pmax, const seren_gpu_params* prm) {
  if (!out || !prm || pmax <= 0 || pmax > (int64_t)1 << 30) return SEREN_GPU_ERR_ARG;
  if (prm->ndim != 3 || prm->leafmax != LEAFMAX || prm->lmax < 1 || prm->lmax > 30 ||
      (prm->kernel != 0 && prm->kernel != 1) || prm->visc != 0 || prm->pp_limit < 1 ||
      prm->pp_gather < 1 || (prm->index_base != 0 && prm->index_base != 1))
    return SEREN_GPU_ERR_ARG;
  seren_oracle* o = new seren_oracle();
  o->prm = *prm;
  o->pmax = pmax;
  o->cmax = (int)(2 * pmax);
  make_tables(prm->kernel, o->tab);
  *out = o;
  return SEREN_GPU_OK;
}

void seren_oracle_destroy(seren_oracle* o) { delete o; }

int seren_oracle_last_error(seren_oracle* o, char* buf, int32_t len) {
  if (!o || !buf || len <= 0) return SEREN_GPU_ERR_ARG;
  std::snprintf(buf, (size_t)len, "%s", o->err.c_str());
  return SEREN_GPU_OK;
}

int seren_oracle_tree_update(seren_oracle* o, int32_t ptot, double* parray, int32_t do_build,
                             int32_t do_reorder, int32_t* perm_out) {
  if (!o || !parray || ptot < 1) return SEREN_GPU_ERR_ARG;
  if (ptot > o->pmax) return o->fail(SEREN_GPU_ERR_CAPACITY, "ptot > pmax");
  for (int64_t i = 0; i < (int64_t)ptot * 6; ++i)
    if (!std::isfinite(parray[i])) return o->fail(SEREN_GPU_ERR_NONFINITE, "non-finite parray");
  if (!do_build && (!o->have_tree || ptot != o->ptot))
    return o->fail(SEREN_GPU_ERR_STATE, "restock without a tree of this size");
  auto t0 = clk::now();
  const bool resized = ptot != o->ptot;
  o->ptot = ptot;
  o->parray.assign(parray, parray + (size_t)ptot * 6);
  if (resized || o->v.size() != (size_t)ptot * 3) {
    o->v.assign((size_t)ptot * 3, 0.0);
    o->rho.assign(ptot, 1.0); o->omega.assign(ptot, 1.0); o->div_v.assign(ptot, 0.0);
    o->drhodt.assign(ptot, 0.0); o->press.assign(ptot, 0.0); o->sound.assign(ptot, 0.0);
    o->pptot.assign(ptot, 0); o->pplist.assign((size_t)ptot * o->prm.pp_limit, 0);
  }
  std::vector<int> dummylist;
  if (do_build) {
    int rc = o->build();
    if (rc) return rc;
    if (do_reorder) {
      o->reorder(dummylist);
      std::memcpy(parray, o->parray.data(), sizeof(double) * (size_t)ptot * 6);
    }
  }
  if (perm_out) {
    for (int i = 0; i < ptot; ++i)
      perm_out[i] = (do_build && do_reorder ? dummylist[i] : i) + o->base();
  }
  o->grav_stock();
  o->copy_to_hydro();
  o->hydro_stock();
  o->stage[0] = secs(t0, clk::now());
  return SEREN_GPU_OK;
}

int seren_oracle_sph_update(seren_oracle* o, int32_t ptot, const int32_t* acclist, int32_t nacc,
                            double* parray, const double* v, double* rho, double* omega,
                            double* div_v, double* drhodt, int32_t* pptot, int32_t* pplist,
                            int32_t first_call) {
  if (!o || !v || ptot != o->ptot || !o->have_tree) return SEREN_GPU_ERR_STATE;
  std::vector<int> act = o->active_list(acclist, nacc);
  if (!o->active_ok(act)) return o->fail(SEREN_GPU_ERR_ARG, "acclist id out of range");
  o->v.assign(v, v + (size_t)ptot * 3);
  o->cnt = seren_oracle_counts{};
  auto t0 = clk::now();
  if (first_call) o->hguess();
  int rc_all = SEREN_GPU_OK;
  seren_oracle_counts tot{};
#pragma omp parallel
  {
    std::vector<int> potlist;
    potlist.reserve(LISTSIZE);
    seren_oracle_counts lc{};
#pragma omp for schedule(dynamic, 64)
    for (int i = 0; i < (int)act.size(); ++i) {
      int rc = o->all_sph_gradh(act[i], potlist, lc);
      if (rc) {
#pragma omp critical
        rc_all = rc;
      }
    }
#pragma omp critical
    {
      tot.gradh_tests += lc.gradh_tests; tot.gradh_pairs += lc.gradh_pairs;
      tot.gradh_passes += lc.gradh_passes; tot.gradh_walks += lc.gradh_walks;
      tot.gradh_final_tests += lc.gradh_final_tests; tot.gradh_final_pairs += lc.gradh_final_pairs;
      tot.gradh_bisections += lc.gradh_bisections;
    }
  }
  if (rc_all) return rc_all;
  o->cnt.gradh_tests = tot.gradh_tests; o->cnt.gradh_pairs = tot.gradh_pairs;
  o->cnt.gradh_passes = tot.gradh_passes; o->cnt.gradh_walks = tot.gradh_walks;
  o->cnt.gradh_final_tests = tot.gradh_final_tests; o->cnt.gradh_final_pairs = tot.gradh_final_pairs;
  o->cnt.gradh_bisections = tot.gradh_bisections;
  auto t1 = clk::now();
  o->update_hmax();
  auto t2 = clk::now();
  o->get_neib_all(act, o->cnt);
  auto t3 = clk::now();
  o->stage[1] = secs(t0, t1); o->stage[2] = secs(t1, t2); o->stage[3] = secs(t2, t3);
  const int L = o->prm.pp_limit;
  for (int p : act) {
    if (parray) { parray[p * 6 + 4] = o->parray[p * 6 + 4]; parray[p * 6 + 5] = o->parray[p * 6 + 5]; }
    if (rho) rho[p] = o->rho[p];
    if (omega) omega[p] = o->omega[p];
    if (div_v) div_v[p] = o->div_v[p];
    if (drhodt) drhodt[p] = o->drhodt[p];
    if (pptot) pptot[p] = o->pptot[p];
    if (pplist && o->pptot[p] <= L)
      for (int k = 0; k < o->pptot[p]; ++k) pplist[(size_t)p * L + k] = o->pplist[(size_t)p * L + k] + o->base();
  }
  if (first_call && parray)
    for (int p = 0; p < ptot; ++p) parray[p * 6 + 4] = o->parray[p * 6 + 4];
  return SEREN_GPU_OK;
}

int seren_oracle_get_neib(seren_oracle* o, int32_t ptot, const int32_t* acclist, int32_t nacc,
                          const double* h, int32_t* pptot, int32_t* pplist) {
  if (!o || ptot != o->ptot || !o->have_tree) return SEREN_GPU_ERR_STATE;
  std::vector<int> act = o->active_list(acclist, nacc);
  if (!o->active_ok(act)) return o->fail(SEREN_GPU_ERR_ARG, "acclist id out of range");
  if (h) for (int p = 0; p < ptot; ++p) o->parray[p * 6 + 4] = h[p];
  o->cnt = seren_oracle_counts{};
  o->update_hmax();
  o->get_neib_all(act, o->cnt);
  const int L = o->prm.pp_limit;
  for (int p : act) {
    if (pptot) pptot[p] = o->pptot[p];
    if (pplist && o->pptot[p] <= L)
      for (int k = 0; k < o->pptot[p]; ++k) pplist[(size_t)p * L + k] = o->pplist[(size_t)p * L + k] + o->base();
  }
  return SEREN_GPU_OK;
}

int seren_oracle_h_gather(seren_oracle* o, int32_t ptot, const int32_t* acclist, int32_t nacc,
                          double* parray) {
  if (!o || !parray || ptot != o->ptot || !o->have_tree) return SEREN_GPU_ERR_STATE;
  std::vector<int> act = o->active_list(acclist, nacc);
  if (!o->active_ok(act)) return o->fail(SEREN_GPU_ERR_ARG, "acclist id out of range");
  std::vector<double> hnew(act.size());
  int rc_all = SEREN_GPU_OK;
  int64_t nodes = 0;
#pragma omp parallel for schedule(dynamic, 64) reduction(+ : nodes)
  for (int i = 0; i < (int)act.size(); ++i) {
    double h = o->parray[act[i] * 6 + 4];
    const int rc = o->h_gather(act[i], h, nodes);
    if (rc) {
#pragma omp critical
      rc_all = rc;
    }
    hnew[i] = h;
  }
  if (rc_all) return o->fail(rc_all, "fewer than pp_gather neighbours (h_gather)");
  for (size_t i = 0; i < act.size(); ++i) {
    o->parray[act[i] * 6 + 4] = hnew[i];
    parray[act[i] * 6 + 4] = hnew[i];
  }
  o->update_hmax();                      // sph_update.F90:121-124
  return SEREN_GPU_OK;
}

int seren_oracle_hydro_forces(seren_oracle* o, const int32_t* acclist, int32_t nacc,
                              const double* press, const double* sound, double* a) {
  if (!o || !press || !sound || !a || !o->have_tree) return SEREN_GPU_ERR_STATE;
  std::vector<int> act = o->active_list(acclist, nacc);
  if (!o->active_ok(act)) return o->fail(SEREN_GPU_ERR_ARG, "acclist id out of range");
  const int ptot = o->ptot;
  o->press.assign(press, press + ptot);
  o->sound.assign(sound, sound + ptot);
  auto t0 = clk::now();
  int64_t npair = 0, nvisc = 0;
#pragma omp parallel reduction(+ : npair, nvisc)
  {
    std::vector<int> pot, lst;
#pragma omp for schedule(dynamic, 64)
    for (int i = 0; i < (int)act.size(); ++i) {
      const int p = act[i];
      double out[3];
      o->hydro_gradh(p, pot, lst, out, npair, nvisc);
      for (int k = 0; k < 3; ++k) a[p * 3 + k] = out[k];
    }
  }
  o->cnt.hydro_pairs = npair;
  o->cnt.hydro_visc = nvisc;
  o->stage[4] = secs(t0, clk::now());
  return SEREN_GPU_OK;
}

int seren_oracle_grav_forces(seren_oracle* o, const int32_t* acclist, int32_t nacc, double* a,
                             double* gpot, int32_t nsink, const double* sink_rmh) {
  if (!o || !a || !gpot || !o->have_tree) return SEREN_GPU_ERR_STATE;
  if (nsink < 0 || (nsink > 0 && !sink_rmh)) return SEREN_GPU_ERR_ARG;
  std::vector<int> act = o->active_list(acclist, nacc);
  if (!o->active_ok(act)) return o->fail(SEREN_GPU_ERR_ARG, "acclist id out of range");
  auto t0 = clk::now();
  int64_t ncell = 0, npair = 0, nnode = 0;
#pragma omp parallel reduction(+ : ncell, npair, nnode)
  {
    std::vector<int> treelist(GLISTSIZE);
#pragma omp for schedule(dynamic, 64)
    for (int i = 0; i < (int)act.size(); ++i) {
      const int p = act[i];
      const double* rp = &o->parray[p * 6];
      double ag[3], pot;
      o->bhgrav_accel(p, 1.0 / rp[4], rp, ag, pot, treelist, ncell, npair, nnode);
      for (int k = 0; k < 3; ++k) a[p * 3 + k] = a[p * 3 + k] + ag[k];
      gpot[p] = pot;
      if (nsink > 0) {
        o->direct_sink_gravity(-1, rp[4], rp, nsink, sink_rmh, ag, pot);
        for (int k = 0; k < 3; ++k) a[p * 3 + k] = a[p * 3 + k] + ag[k];
        gpot[p] = gpot[p] + pot;
      }
    }
  }
  o->cnt.grav_cells = ncell;
  o->cnt.grav_pairs = npair;
  o->cnt.grav_nodes = nnode;
  o->stage[5] = secs(t0, clk::now());
  return SEREN_GPU_OK;
}

int seren_oracle_sink_forces(seren_oracle* o, int32_t nsink, const double* sink_rmh,
                             double* sink_a, double* sink_gpot) {
  if (!o || nsink < 1 || !sink_rmh || !sink_a || !sink_gpot || !o->have_tree) return SEREN_GPU_ERR_ARG;
  std::vector<int> treelist(GLISTSIZE);
  int64_t nc = 0, np = 0, nn = 0;
  for (int s = 0; s < nsink; ++s) {
    const double* sr = &sink_rmh[s * 5];
    double ag[3], pot;
    o->bhgrav_accel(-1 - s, 1.0 / sr[4], sr, ag, pot, treelist, nc, np, nn);
    for (int k = 0; k < 3; ++k) sink_a[s * 3 + k] = ag[k];
    sink_gpot[s] = pot;
    o->direct_sink_gravity(s, sr[4], sr, nsink, sink_rmh, ag, pot);
    for (int k = 0; k < 3; ++k) sink_a[s * 3 + k] = sink_a[s * 3 + k] + ag[k];
    sink_gpot[s] = sink_gpot[s] + pot;
  }
  return SEREN_GPU_OK;
}

int seren_oracle_direct_gravity(seren_oracle* o, const int32_t* ids, int32_t n, double* a,
                                double* gpot) {
  if (!o || !ids || n < 0 || !a || !gpot || o->ptot < 1) return SEREN_GPU_ERR_ARG;
  const int ptot = o->ptot;
#pragma omp parallel for schedule(dynamic, 4)
  for (int i = 0; i < n; ++i) {
    const int p = ids[i] - o->base();
    const double* rp = &o->parray[p * 6];
    const double invhp = 1.0 / rp[4];
    const double zo_p = rp[5];
    double ag[3] = {0, 0, 0}, pot = 0.0;
    for (int pp = 0; pp < ptot; ++pp) {
      if (pp == p) continue;
      const double* rpp = &o->parray[pp * 6];
      double at[3], dpot;
      o->gravity_gradh(invhp, rpp[4], rpp[3], rp, rpp, zo_p, rpp[5], at, dpot);
      for (int k = 0; k < 3; ++k) ag[k] = ag[k] + at[k];
      pot = pot + dpot;
    }
    for (int k = 0; k < 3; ++k) a[i * 3 + k] = ag[k];
    gpot[i] = pot;
  }
  return SEREN_GPU_OK;
}

int seren_oracle_tree_export(seren_oracle* o, int32_t* ctot, int32_t* ltot, int32_t* leaf,
                             int32_t* nextcell, int32_t* ifopen, int32_t* plist,
                             int32_t* first_cell, int32_t* last_cell, double* grav_r,
                             double* grav_m, double* grav_q, double* dminsqd, double* hydro_r,
                             double* rmax, double* hrangemax) {
  if (!o || !o->have_tree) return SEREN_GPU_ERR_STATE;
  if (ctot) *ctot = o->ctot;
  if (ltot) *ltot = o->ltot;
  for (int c = 0; c <= o->ctot; ++c) {
    const GravNode& g = o->grav[c];
    const HydroNode& h = o->hyd[c];
    if (leaf) leaf[c] = g.leaf;
    if (nextcell) nextcell[c] = g.nextcell;
    if (ifopen) ifopen[c] = g.leaf > 0 ? -1 : g.ifopen;
    if (plist)
      for (int k = 0; k < LEAFMAX; ++k)
        plist[c * LEAFMAX + k] = (g.leaf > 0 && k < g.leaf) ? g.plist[k] + o->base() : -1;
    if (grav_r) for (int k = 0; k < 3; ++k) grav_r[c * 3 + k] = g.r[k];
    if (grav_m) grav_m[c] = g.m;
    if (grav_q) for (int k = 0; k < 5; ++k) grav_q[c * 5 + k] = g.q[k];
    if (dminsqd) dminsqd[c] = g.dminsqd;
    if (hydro_r) for (int k = 0; k < 3; ++k) hydro_r[c * 3 + k] = h.r[k];
    if (rmax) rmax[c] = h.rmax;
    if (hrangemax) hrangemax[c] = h.hrangemax;
  }
  for (int l = 0; l <= o->ltot; ++l) {
    if (first_cell) first_cell[l] = o->first_cell[l];
    if (last_cell) last_cell[l] = o->last_cell[l];
  }
  return SEREN_GPU_OK;
}

int seren_oracle_get_counts(seren_oracle* o, seren_oracle_counts* out) {
  if (!o || !out) return SEREN_GPU_ERR_ARG;
  *out = o->cnt;
  return SEREN_GPU_OK;
}

int seren_oracle_stage_seconds(seren_oracle* o, double* sec) {
  if (!o || !sec) return SEREN_GPU_ERR_ARG;
  for (int i = 0; i < 6; ++i) sec[i] = o->stage[i];
  return SEREN_GPU_OK;
}

}  // extern "C"
