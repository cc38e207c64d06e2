// Post-SCF geometric corrections on the device, in kcal/mol: D2-style dispersion
// (pm7-rs src/dispersion.rs:186-284 and the smooth variant :147-184,383-426), the
// EH+ hydrogen-bond term (src/hbond.rs:53-760,1294-1321, molecular path), the C#C
// and Si-O-H molecular-mechanics terms (src/mm_corrections.rs) and PM7-HH's H-H
// repulsion (src/hh_rep.rs). Each term is a per-item kernel whose values are summed
// in a fixed order.
#include <cuda_runtime.h>

#include <vector>

#include "common.cuh"
#include "batch.hpp"
#include "engine_internal.hpp"
#include "gradient.cuh"
#include "kernels.hpp"

namespace pm7 {
namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr double kMopacTwoPi = 6.28318530717959;

__device__ double c6_of(int z) {
  switch (z) {
    case 1: return 0.16; case 2: return 0.084; case 5: return 5.79; case 6: return 1.65; case 7: return 1.11;
    case 8: return 0.70; case 9: return 0.57; case 10: return 0.45; case 15: return 3.25; case 16: return 5.79;
    case 17: return 5.97; case 18: return 3.71; case 27: return 0.04; case 35: return 11.60; case 36: return 4.47;
    case 53: return 25.80; case 54: return 16.50; default: return 0.0;
  }
}
__device__ double r0_of(int z) {
  switch (z) {
    case 1: return 156.0; case 2: return 140.0; case 5: return 180.0; case 6: return 170.0; case 7: return 155.0;
    case 8: return 152.0; case 9: return 147.0; case 10: return 154.0; case 15: return 180.0; case 16: return 180.0;
    case 17: return 175.0; case 18: return 188.0; case 28: return 140.0; case 35: return 185.0; case 36: return 202.0;
    case 53: return 198.0; case 54: return 216.0; default: return 0.0;
  }
}
__device__ double neff_of(int z) {
  switch (z) {
    case 1: return 0.80; case 2: return 1.42; case 5: return 2.16; case 6: return 2.50; case 7: return 2.82;
    case 8: return 3.15; case 9: return 3.48; case 10: return 3.81; case 15: return 4.50; case 16: return 4.80;
    case 17: return 5.10; case 18: return 5.40; case 27: return 2.90; case 35: return 6.00; case 36: return 6.30;
    case 53: return 6.95; case 54: return 7.25; default: return 0.0;
  }
}
__device__ bool disp_params(int z) { return z >= 1 && z <= 86 && c6_of(z) != 0.0 && r0_of(z) != 0.0 && neff_of(z) != 0.0; }

__constant__ double kCovalent[87] = {
    0.0,  0.31, 0.28, 1.28, 0.96, 0.84, 0.76, 0.71, 0.66, 0.57, 0.58, 1.66, 1.41, 1.21, 1.11, 1.07, 1.05, 1.02,
    1.06, 2.03, 1.76, 1.70, 1.60, 1.53, 1.39, 1.39, 1.32, 1.26, 1.24, 1.32, 1.22, 1.22, 1.20, 1.19, 1.20, 1.20,
    1.16, 2.20, 1.95, 1.90, 1.75, 1.64, 1.54, 1.47, 1.46, 1.42, 1.39, 1.45, 1.44, 1.42, 1.39, 1.39, 1.38, 1.39,
    1.40, 2.44, 2.15, 2.07, 2.04, 2.03, 2.01, 1.99, 1.98, 1.98, 1.96, 1.94, 1.92, 1.92, 1.89, 1.90, 1.87, 1.87,
    1.75, 1.70, 1.62, 1.51, 1.44, 1.41, 1.36, 1.36, 1.32, 1.45, 1.46, 1.48, 1.40, 1.50, 1.50};
__device__ double covalent(int z) { return (z >= 0 && z < 87) ? kCovalent[z] : 1.5; }

// MOPAC covrad (Angstrom) scaled by 4/3, for the EH+ bonding test.
__constant__ double kCovrad[94] = {
    0.32, 0.46, 1.20, 0.94, 0.77, 0.75, 0.71, 0.63, 0.64, 0.67, 1.40, 1.25, 1.13, 1.04, 1.10, 1.02, 0.99, 0.96, 1.76,
    1.54, 1.33, 1.22, 1.21, 1.10, 1.07, 1.04, 1.00, 0.99, 1.01, 1.09, 1.12, 1.09, 1.15, 1.10, 1.14, 1.17, 1.89, 1.67,
    1.47, 1.39, 1.32, 1.24, 1.15, 1.13, 1.13, 1.08, 1.15, 1.23, 1.28, 1.26, 1.26, 1.23, 1.32, 1.31, 2.09, 1.76, 1.62,
    1.47, 1.58, 1.57, 1.56, 1.55, 1.51, 1.52, 1.51, 1.50, 1.49, 1.49, 1.48, 1.53, 1.46, 1.37, 1.31, 1.23, 1.18, 1.16,
    1.11, 1.12, 1.13, 1.32, 1.30, 1.30, 1.36, 1.31, 1.38, 1.42, 2.01, 1.81, 1.67, 1.58, 1.52, 1.53, 1.54, 1.55};
__device__ double covrad43(int z) { return (z <= 0 || z > 94) ? 1.5 * 4.0 / 3.0 : kCovrad[z - 1] * 4.0 / 3.0; }

__device__ __forceinline__ double3 pos_ang(const double *xyz, int i) {
  return make_double3(xyz[3 * i] * kA0, xyz[3 * i + 1] * kA0, xyz[3 * i + 2] * kA0);
}
__device__ __forceinline__ double dist_ang(const double *xyz, int a, int b) {
  const double3 p = pos_ang(xyz, a), q = pos_ang(xyz, b);
  const double dx = p.x - q.x, dy = p.y - q.y, dz = p.z - q.z;
  return sqrt(dx * dx + dy * dy + dz * dz);
}
__device__ __forceinline__ double dist2_ang(const double *xyz, int a, int b) {
  const double3 p = pos_ang(xyz, a), q = pos_ang(xyz, b);
  const double dx = p.x - q.x, dy = p.y - q.y, dz = p.z - q.z;
  return dx * dx + dy * dy + dz * dz;
}

// Slater-Kirkwood-combined damped C6/R^6 (dispersion.rs:337-364); r in Bohr.
__device__ double pair_dispersion(int zi, int zj, double c6i, double c6j, double r) {
  if (!disp_params(zi) || !disp_params(zj)) return 0.0;
  const double ni = neff_of(zi), nj = neff_of(zj);
  const double c6 = 2.0 * pow(c6i * c6i * c6j * c6j * ni * nj, 1.0 / 3.0) /
                    (pow(c6i * nj * nj, 1.0 / 3.0) + pow(c6j * ni * ni, 1.0 / 3.0));
  const double ri = r0_of(zi), rj = r0_of(zj);
  const double r0 = (ri * ri * ri + rj * rj * rj) / (ri * ri + rj * rj) / 1000.0 * 2.0;
  const double rn = r * (kA0 * 0.1);
  const double damp = exp((rn * (1.0 / (1.226593 * r0)) - 1.0) * (-15.450118)) + 1.0;
  const double r6 = rn * rn * rn * rn * rn * rn;
  return (1.0 / r6) * (c6 / (1000.0 * 4.184)) / damp * (-2.286419);
}

// Per-atom effective C6: discrete neighbour count (MOPAC nbonds) or the smooth one.
__device__ __forceinline__ void c6_atom(int n, const int *__restrict__ z, const double *__restrict__ xyz, int smooth,
                                        double *__restrict__ c6, int i) {
  if (i >= n) return;
  int cnt = 0;
  double scnt = 0.0;
  const double ri = covalent(z[i]);
  for (int j = 0; j < n; ++j) {
    if (j == i) continue;
    const double dx = xyz[3 * j] - xyz[3 * i], dy = xyz[3 * j + 1] - xyz[3 * i + 1], dz = xyz[3 * j + 2] - xyz[3 * i + 2];
    const double r = sqrt(dx * dx + dy * dy + dz * dz);
    const double rc = 1.3 * (ri + covalent(z[j]));
    if (smooth) {
      const double e = exp(-26.0 * (rc / kA0 / r - 1.0));
      scnt += isfinite(e) ? 1.0 / (1.0 + e) : 0.0;
    } else if (r * kA0 < rc) {
      ++cnt;
    }
  }
  if (z[i] != 6) {
    c6[i] = c6_of(z[i]);
  } else if (smooth) {
    const double s = 1.0 / (1.0 + exp(-(scnt - 3.5) * 40.0));
    c6[i] = 1.65 + (0.95 - 1.65) * s;
  } else {
    c6[i] = cnt == 4 ? 0.95 : 1.65;
  }
}

// The pair terms of atoms of numbers zu, zv (C6 coefficients c6u, c6v) at distance r (Bohr):
// dispersion, the C#C switch (counted 12 kcal/mol per full bond by the caller) and PM7-HH.
__device__ __forceinline__ void pair_corr_r(int zu, int zv, double c6u, double c6v, int hh, double r, double &ed,
                                            double &ey, double &eh) {
  ed = pair_dispersion(zu, zv, c6u, c6v, r);
  ey = 0.0;
  eh = 0.0;
  const double ra = r * kA0;
  if (zu == 6 && zv == 6 && ra < 1.33) {
    if (ra < 1.21) {
      ey = 1.0;
    } else {
      const double x = (ra - 1.21) / (1.33 - 1.21);
      const double x3 = x * x * x, x4 = x3 * x, x5 = x4 * x, x6 = x5 * x;
      ey = (1.0 - 10.0 * x3 + 15.0 * x4 - 6.0 * x5) + (-5.0 + 25.0 * x) * (x3 - 3.0 * x4 + 3.0 * x5 - x6);
    }
  }
  if (hh && zu == 1 && zv == 1) {
    if (ra <= 1.0) eh = 25.46293603147693;
    else if (ra < 1.5) {
      const double r2 = ra * ra, r3 = r2 * ra, r4 = r3 * ra, r5 = r4 * ra;
      eh = r5 * (-2714.9523516034697) + r4 * 17103.650110591705 + r3 * (-42511.85798221796) +
           r2 * 52063.19679913834 + ra * (-31430.65833597229) + 7516.08469609514;
    } else {
      eh = exp(pow(ra, 1.72905) * (-1.53965)) * 118.7326;
    }
  }
}

// Pair terms of every u < v: dispersion, C#C and PM7-HH. Grid (ceil(N/128), N).
__device__ __forceinline__ void pair_corr_elem(int n, const int *__restrict__ z, const double *__restrict__ xyz,
                                               const double *__restrict__ c6, int hh, int u, int v, double &ed,
                                               double &ey, double &eh) {
  ed = ey = eh = 0.0;
  if (v > u && v < n) {
    const double dx = xyz[3 * v] - xyz[3 * u], dy = xyz[3 * v + 1] - xyz[3 * u + 1], dz = xyz[3 * v + 2] - xyz[3 * u + 2];
    pair_corr_r(z[u], z[v], c6[u], c6[v], hh, sqrt(dx * dx + dy * dy + dz * dz), ed, ey, eh);
  }
}

// Block sums of one (u, column block) of the pair sweep into partial `slot`.
__device__ __forceinline__ void pair_corr_block(int n, const int *__restrict__ z, const double *__restrict__ xyz,
                                                const double *__restrict__ c6, int hh, int u, int bx, size_t slot,
                                                double *__restrict__ part_disp, double *__restrict__ part_yne,
                                                double *__restrict__ part_hh) {
  double ed, ey, eh;
  pair_corr_elem(n, z, xyz, c6, hh, u, bx * blockDim.x + threadIdx.x, ed, ey, eh);
  const double sd = block_sum<128>(ed);
  const double sy = block_sum<128>(ey);
  const double sh = block_sum<128>(eh);
  if (threadIdx.x == 0) {
    part_disp[slot] = sd;
    part_yne[slot] = sy * 12.0;
    part_hh[slot] = sh;
  }
}

// Si-O-H bending penalty, one thread per oxygen (mm_corrections.rs:154-224).
__device__ __forceinline__ void sioh_atom(int n, const int *__restrict__ z, const double *__restrict__ xyz,
                                          double *__restrict__ e_out, int o) {
  if (o >= n) return;
  double e = 0.0;
  if (z[o] == 8) {
    int si = -1, h = -1;
    double dsi = 0.0, dh = 0.0;
    for (int k = 0; k < n; ++k) {
      if (k == o) continue;
      const double r = dist_ang(xyz, k, o);
      if (z[k] == 14 && r < 2.4 && (si < 0 || r < dsi)) {
        si = k;
        dsi = r;
      }
      if (z[k] == 1 && r < 1.4 && (h < 0 || r < dh)) {
        h = k;
        dh = r;
      }
    }
    if (si >= 0 && h >= 0) {
      const double rso = dsi, roh = dh;
      const double damp = exp(-33.0 * fmax(rso * rso - 1.7 * 1.7, 0.0)) * exp(-68.0 * fmax(roh * roh - 1.0, 0.0));
      const double3 S = pos_ang(xyz, si), O = pos_ang(xyz, o), H = pos_ang(xyz, h);
      const double ux = S.x - O.x, uy = S.y - O.y, uz = S.z - O.z, vx = H.x - O.x, vy = H.y - O.y, vz = H.z - O.z;
      double cs = (ux * vx + uy * vy + uz * vz) / (sqrt(ux * ux + uy * uy + uz * uz) * sqrt(vx * vx + vy * vy + vz * vz));
      cs = fmin(fmax(cs, -1.0), 1.0);
      const double ang = acos(cs), ref = 125.0 * kPi / 180.0;
      e = 15.0 * damp * (ang - ref) * (ang - ref);
    }
  }
  e_out[o] = e;
}

// ---- EH+ hydrogen bonds ------------------------------------------------------

__device__ double bangle(const double *xyz, int i, int j, int k) {
  const double d2ij = dist2_ang(xyz, i, j), d2jk = dist2_ang(xyz, j, k), d2ik = dist2_ang(xyz, i, k);
  const double xy = sqrt(d2ij * d2jk);
  if (xy < 1.0e-20) return 0.0;
  return acos(fmin(fmax(0.5 * (d2ij + d2jk - d2ik) / xy, -1.0), 1.0));
}

__device__ double dang(double a1, double a2, double b1, double b2) {
  const double zero = 1.0e-6;
  if ((fabs(a1) >= zero || fabs(a2) >= zero) && (fabs(b1) >= zero || fabs(b2) >= zero)) {
    const double an = 1.0 / sqrt(a1 * a1 + a2 * a2), bn = 1.0 / sqrt(b1 * b1 + b2 * b2);
    a1 *= an;
    a2 *= an;
    b1 *= bn;
    b2 *= bn;
    const double sinth = a1 * b2 - a2 * b1;
    double rcos = acos(fmin(fmax(a1 * b1 + a2 * b2, -1.0), 1.0));
    if (fabs(rcos) >= 4.0e-5) {
      if (sinth > 0.0) rcos = kMopacTwoPi - rcos;
      return -rcos;
    }
  }
  return 0.0;
}

__device__ double dihed(const double *xyz, int i, int j, int k, int l) {
  const double3 I = pos_ang(xyz, i), J = pos_ang(xyz, j), K = pos_ang(xyz, k), L = pos_ang(xyz, l);
  const double xi1 = I.x - K.x, xj1 = J.x - K.x, xl1 = L.x - K.x;
  const double yi1 = I.y - K.y, yj1 = J.y - K.y, yl1 = L.y - K.y;
  const double zi1 = I.z - K.z, zj1 = J.z - K.z, zl1 = L.z - K.z;
  const double d = sqrt(xj1 * xj1 + yj1 * yj1 + zj1 * zj1);
  const double cosa = d > 0.0 ? fmin(fmax(zj1 / d, -1.0), 1.0) : 0.0;
  const double ddd = 1.0 - cosa * cosa;
  const double yxd = ddd > 0.0 ? d * sqrt(ddd) : 0.0;
  double xi2 = xi1, xl2 = xl1, yi2 = yi1, yl2 = yl1, sinth = 0.0;
  if (ddd > 0.0 && yxd > 1.0e-6) {
    const double cosph = yj1 / yxd, sinph = xj1 / yxd;
    xi2 = xi1 * cosph - yi1 * sinph;
    xl2 = xl1 * cosph - yl1 * sinph;
    yi2 = xi1 * sinph + yi1 * cosph;
    const double yj2 = xj1 * sinph + yj1 * cosph;
    yl2 = xl1 * sinph + yl1 * cosph;
    sinth = yj2 / d;
  }
  const double yi3 = yi2 * cosa - zi1 * sinth, yl3 = yl2 * cosa - zl1 * sinth;
  double angle = dang(xl2, yl3, xi2, yi3);
  if (angle < 0.0) angle += 2.0 * kPi;
  if (angle >= kMopacTwoPi) angle = 0.0;
  return angle;
}

__device__ __forceinline__ double bonding(const int *z, int x, int y) { return covrad43(z[x]) + covrad43(z[y]); }

// Covalent neighbours (ascending scan, at most 4: a fifth evicts the longest).
__device__ __forceinline__ void hb_neighbours_atom(int n, const int *__restrict__ z, const double *__restrict__ xyz,
                                                   int *__restrict__ nbr, int *__restrict__ nbc, int a) {
  if (a >= n) return;
  int list[5];
  int cnt = 0;
  for (int j = 0; j < n; ++j) {
    if (j == a || !(dist_ang(xyz, j, a) < bonding(z, j, a))) continue;
    list[cnt++] = j;
    if (cnt == 5) {
      int worst = 0;
      double wd = -1.0;
      for (int q = 0; q < 5; ++q) {
        const double dd = dist_ang(xyz, a, list[q]);
        if (dd > wd) {
          wd = dd;
          worst = q;
        }
      }
      for (int q = worst; q < 4; ++q) list[q] = list[q + 1];
      cnt = 4;
    }
  }
  for (int q = 0; q < 4; ++q) nbr[4 * a + q] = q < cnt ? list[q] : -1;
  nbc[a] = cnt;
}

__device__ __forceinline__ double wrap_pi(double v) {
  if (v <= -kPi) v += 2.0 * kPi;
  if (v > kPi) v -= 2.0 * kPi;
  return v;
}

// Reference atoms of one side (hbond.rs:439-505): slots r1, r2, r3.
__device__ void assign_refs(int n, const int *z, const double *xyz, const int *nb, int nbn, int x, int h, int &r1,
                            int &r2, int &r3) {
  const int fill = dist_ang(xyz, x, h) < bonding(z, x, h) ? h : x;
  if (nbn == 3 || nbn == 4) {
    int o[4];
    for (int q = 0; q < nbn; ++q) o[q] = nb[q];
    // stable descending sort by distance from h
    for (int a = 1; a < nbn; ++a) {
      const int key = o[a];
      const double kd = dist_ang(xyz, key, h);
      int b = a - 1;
      while (b >= 0 && dist_ang(xyz, o[b], h) < kd) {
        o[b + 1] = o[b];
        --b;
      }
      o[b + 1] = key;
    }
    r1 = o[0];
    r2 = o[1];
    r3 = o[2];
  } else if (nbn == 2) {
    if (dist_ang(xyz, nb[0], h) >= dist_ang(xyz, nb[1], h)) {
      r1 = nb[0];
      r2 = nb[1];
    } else {
      r1 = nb[1];
      r2 = nb[0];
    }
    r3 = fill;
  } else if (nbn == 1) {
    r1 = nb[0];
    int best = nb[0];
    double bd = -1.0;
    for (int k = 0; k < n; ++k) {
      if (k == nb[0] || !(dist_ang(xyz, k, nb[0]) < bonding(z, k, nb[0]))) continue;
      const double dd = dist_ang(xyz, k, h);
      if (dd > bd) {
        bd = dd;
        best = k;
      }
    }
    r2 = best;
    r3 = fill;
  } else {
    r1 = r2 = r3 = fill;
  }
}

__device__ __forceinline__ double deg(double d) { return kPi / (180.0 / d); }

// side_terms (hbond.rs:627-743); returns false on a hard cut-off.
__device__ bool side_terms(const int *z, const double *xyz, int nrb, int heavy, int r1, int r2, int r3, int h,
                           double &a2c_out, double &tc_out) {
  double a2s = 0.0, a2s2 = 0.0, ts = 0.0;
  bool tcs = false, tcs2 = false;
  if (z[heavy] == 8) {
    if (nrb == 1) {
      a2s = kPi;
      a2s2 = deg(120.0);
      tcs2 = true;
    } else {
      a2s = deg(109.48);
      a2s2 = a2s;
      ts = deg(54.74);
    }
  } else if (z[heavy] == 7) {
    if (nrb == 2) {
      a2s = deg(120.0);
      a2s2 = a2s;
    } else {
      a2s = deg(109.48);
      a2s2 = a2s;
      ts = deg(54.74);
      tcs = true;
    }
  }
  double tcheck = 0.0;
  if (tcs) {
    double tc = dihed(xyz, r2, r1, heavy, r3);
    if (tc <= -kPi) tc += 2.0 * kPi;
    if (tc > kPi) tc -= 2.0 * kPi;
    tc = tc < 0.0 ? -kPi - tc : kPi - tc;
    const double bac = tc;
    double tcp = tc < 0.0 ? -tc : tc;
    tcp *= 180.0 / kPi;
    ts += deg((54.74 - tcp) / 54.74 * 35.26);
    a2s -= deg((54.74 - tcp) / 54.74 * 19.48);
    a2s2 = a2s;
    tcheck = bac;
  }
  const double ang2 = bangle(xyz, r1, heavy, h);
  double a2c = cos(a2s - ang2);
  const double a2c2 = cos(a2s2 - ang2);
  if (a2c2 > a2c) a2c = a2c2;
  if (a2c <= 0.0) return false;
  double tcorr = dihed(xyz, r2, r1, heavy, h);
  if (tcorr <= -kPi) tcorr += 2.0 * kPi;
  if (tcorr > kPi) tcorr -= 2.0 * kPi;
  if (!tcs2 || fabs(tcorr * 180.0 / kPi) > 90.0) tcorr = tcorr < 0.0 ? -kPi - tcorr : kPi - tcorr;
  double tcos;
  if (tcheck < 0.0) tcos = cos(wrap_pi(ts - tcorr));
  else if (tcheck > 0.0) tcos = cos(wrap_pi(-ts - tcorr));
  else {
    const double c1 = cos(wrap_pi(ts - tcorr)), c2 = cos(wrap_pi(-ts - tcorr));
    tcos = c2 > c1 ? c2 : c1;
  }
  if (dist_ang(xyz, h, heavy) > dist_ang(xyz, h, r1) && tcs2) tcos = 0.0;
  if (r2 == r3 || h == r3) tcos = 1.0;
  a2c_out = a2c;
  tc_out = tcos;
  return true;
}

// EH+ energy of donor a1 - hydrogen h ... acceptor a5 (hbond.rs:263-406 topology,
// :525-620 energy).
__device__ double eh_plus(int n, const int *z, const double *xyz, const int *nbr, const int *nbc, int a1, int h,
                          int a5) {
  const int *na = nbr + 4 * a1, *nb = nbr + 4 * a5;
  const int nra = nbc[a1], nrb = nbc[a5];
  for (int p = 0; p < nra; ++p) {
    if (na[p] == a5) return 0.0;
    for (int q = 0; q < nrb; ++q)
      if (na[p] == nb[q] && nb[q] != h) return 0.0;  // 1-3 / 1-4 contact: disabled
  }
  int s2, s3, s4, s6, s7, s8;
  assign_refs(n, z, xyz, na, nra, a1, h, s2, s3, s4);
  assign_refs(n, z, xyz, nb, nrb, a5, h, s6, s7, s8);
  const double a0 = kA0;
  const double sn3 = -0.171271 * a0 * a0, so3 = -0.098822 * a0 * a0, sn2 = -0.171271 * a0 * a0, so2 = so3;
  const double hartree2kcal = kEv * kEvToKcal;
  const double angle_cos = -cos(bangle(xyz, a1, h, a5));
  if (angle_cos <= 0.0) return 0.0;
  double a2c, tc, a2cn, tcn;
  if (!side_terms(z, xyz, nra, a1, s2, s3, s4, h, a2c, tc)) return 0.0;
  if (!side_terms(z, xyz, nrb, a5, s6, s7, s8, h, a2cn, tcn)) return 0.0;
  tcn = fabs(tcn);
  const double sa = z[a1] == 7 ? (nra >= 3 ? sn3 : sn2) : (nra >= 2 ? so3 : so2);
  const double sb = z[a5] == 7 ? (nrb >= 3 ? sn3 : sn2) : (nrb >= 2 ? so3 : so2);
  const double sc = (sa + sb) / 2.0;
  const double had = dist_ang(xyz, h, a1), hbd = dist_ang(xyz, h, a5);
  const double xmin = fmin(had, hbd), gap = fmax(had, hbd) - xmin;
  double damping = gap > 0.5 ? 1.0 - 1.0 / (1.0 + exp(-60.0 * (xmin / 1.2 - 1.0))) : 1.0;
  const double oo = dist_ang(xyz, a1, a5);
  damping /= 1.0 + exp(-100.0 * (oo / 2.4 - 1.0));
  damping *= 1.0 - 1.0 / (1.0 + exp(-10.0 * (oo / 7.0 - 1.0)));
  const double inner = 1.0 - a2c * tc * a2cn * tcn;
  double e = sc / (oo * oo) * (angle_cos * angle_cos) * (1.0 - inner * inner) * hartree2kcal * damping;
  if (z[a1] == 8 && z[a5] == 8) {
    const double t = fmax(oo - 2.67, 0.0);
    e += -2.5 * exp(-80.0 * t * t) * (angle_cos * angle_cos * angle_cos * angle_cos);
  }
  return e;
}

__device__ __forceinline__ bool is_acceptor(int z) { return z == 7 || z == 8; }

// Whether acceptor k forms an H-bond term with donor di and hydrogen j (hbond.rs:263-406): an
// N or O within 7 A of the donor, D-H...A angle above 90 degrees, and not a second donor of j
// of lower index (that pair is taken as (k, j, di)).
__device__ __forceinline__ bool hb_acceptor_ok(const int *z, const double *xyz, int j, int di, int k) {
  if (k == di || !is_acceptor(z[k])) return false;
  if (!(dist2_ang(xyz, k, di) < 7.0 * 7.0)) return false;
  if (bangle(xyz, k, j, di) <= kPi * 0.5) return false;
  if (k < di && dist2_ang(xyz, k, j) < 1.4 * 1.4) return false;  // already taken as (k, j, di)
  return true;
}

// One warp per hydrogen j: every donor i (N/O within 1.4 A of j, in atom order) and
// acceptor k (N/O within 7 A of i, D-H...A angle above 90 degrees, lanes over k), each
// unordered {i,k} once with the lower-index donor taking the bond as in the reference's
// scan; lane sums are combined in a fixed shuffle order.
__device__ __forceinline__ void hbonds_warp(int n, const int *__restrict__ z, const double *__restrict__ xyz,
                                            const int *__restrict__ nbr, const int *__restrict__ nbc,
                                            double *__restrict__ e_out, int j) {
  const int lane = threadIdx.x & 31;
  if (j >= n) return;
  double e = 0.0;
  if (z[j] == 1) {
    const double rah2 = 1.4 * 1.4;
    for (int base = 0; base < n; base += 32) {
      const int i = base + lane;
      const bool donor = i < n && is_acceptor(z[i]) && dist2_ang(xyz, i, j) < rah2;
      unsigned m = __ballot_sync(0xffffffffu, donor);
      while (m) {
        const int di = base + __ffs(m) - 1;
        m &= m - 1;
        for (int k = lane; k < n; k += 32)
          if (hb_acceptor_ok(z, xyz, j, di, k)) e += eh_plus(n, z, xyz, nbr, nbc, di, j, k);
      }
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) e += __shfl_down_sync(0xffffffffu, e, o);
  if (lane == 0) e_out[j] = e;
}

__device__ __forceinline__ void finish_block(int n_pairs_part, const double *__restrict__ pd,
                                             const double *__restrict__ py, const double *__restrict__ ph, int n,
                                             const double *__restrict__ ehb, const double *__restrict__ esioh,
                                             double *__restrict__ out) {
  double s0 = 0, s1 = 0, s2 = 0, s3 = 0, s4 = 0;
  for (int i = threadIdx.x; i < n_pairs_part; i += 256) {
    s0 += pd[i];
    s2 += py[i];
    s4 += ph[i];
  }
  for (int i = threadIdx.x; i < n; i += 256) {
    s1 += ehb[i];
    s3 += esioh[i];
  }
  s0 = block_sum<256>(s0);
  s1 = block_sum<256>(s1);
  s2 = block_sum<256>(s2);
  s3 = block_sum<256>(s3);
  s4 = block_sum<256>(s4);
  if (threadIdx.x == 0) {
    out[0] = s0;
    out[1] = s1;
    out[2] = s2;
    out[3] = s3;
    out[4] = s4;
  }
}

// Scratch of one molecule's corrections (corrections_scratch floats of layout below).
struct CorrView {
  int n, gx;
  size_t parts;
  double *pd, *py, *ph, *c6, *ehb, *esioh;
  int *nbr, *nbc;
};
__host__ __device__ inline CorrView corr_view(int n, double *scratch) {
  CorrView v;
  v.n = n;
  v.gx = (n + 127) / 128;
  v.parts = (size_t)v.gx * n;
  v.pd = scratch;
  v.py = v.pd + v.parts;
  v.ph = v.py + v.parts;
  v.c6 = v.ph + v.parts;
  v.ehb = v.c6 + n;
  v.esioh = v.ehb + n;
  v.nbr = reinterpret_cast<int *>(v.esioh + n);
  v.nbc = v.nbr + 4 * n;
  return v;
}

// ---- one molecule ----
__global__ void k_c6(int n, const int *__restrict__ z, const double *__restrict__ xyz, int smooth,
                     double *__restrict__ c6) {
  c6_atom(n, z, xyz, smooth, c6, blockIdx.x * blockDim.x + threadIdx.x);
}
__global__ void k_pair_corr(int n, const int *__restrict__ z, const double *__restrict__ xyz,
                            const double *__restrict__ c6, int hh, double *__restrict__ part_disp,
                            double *__restrict__ part_yne, double *__restrict__ part_hh) {
  pair_corr_block(n, z, xyz, c6, hh, blockIdx.y, blockIdx.x, (size_t)blockIdx.y * gridDim.x + blockIdx.x, part_disp,
                  part_yne, part_hh);
}
__global__ void k_sioh(int n, const int *__restrict__ z, const double *__restrict__ xyz, double *__restrict__ e_out) {
  sioh_atom(n, z, xyz, e_out, blockIdx.x * blockDim.x + threadIdx.x);
}
// A warp per atom i: the discrete covalent-neighbour count (an integer, so the lanes' order
// does not matter) and the C6 it selects -- c6_atom's discrete branch.
__global__ void k_c6_discrete_warp(int n, const int *__restrict__ z, const double *__restrict__ xyz,
                                   double *__restrict__ c6) {
  const int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (i >= n) return;
  int cnt = 0;
  const double ri = covalent(z[i]);
  for (int j = lane; j < n; j += 32) {
    if (j == i) continue;
    const double dx = xyz[3 * j] - xyz[3 * i], dy = xyz[3 * j + 1] - xyz[3 * i + 1], dz = xyz[3 * j + 2] - xyz[3 * i + 2];
    const double r = sqrt(dx * dx + dy * dy + dz * dz);
    const double rc = 1.3 * (ri + covalent(z[j]));
    if (r * kA0 < rc) ++cnt;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
  if (lane == 0) c6[i] = z[i] != 6 ? c6_of(z[i]) : (cnt == 4 ? 0.95 : 1.65);
}

// A warp per atom a: hb_neighbours_atom's ascending scan (a fifth neighbour evicts the longest),
// candidates found 32 at a time and taken in ascending order by every lane alike.
__global__ void k_hb_neighbours_warp(int n, const int *__restrict__ z, const double *__restrict__ xyz,
                                     int *__restrict__ nbr, int *__restrict__ nbc) {
  const int a = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (a >= n) return;
  int list[5];
  int cnt = 0;
  for (int base = 0; base < n; base += 32) {
    const int j = base + lane;
    const bool cand = j < n && j != a && dist_ang(xyz, j, a) < bonding(z, j, a);
    unsigned m = __ballot_sync(0xffffffffu, cand);
    while (m) {
      list[cnt++] = base + __ffs(m) - 1;
      m &= m - 1;
      if (cnt == 5) {
        int worst = 0;
        double wd = -1.0;
        for (int q = 0; q < 5; ++q) {
          const double dd = dist_ang(xyz, a, list[q]);
          if (dd > wd) {
            wd = dd;
            worst = q;
          }
        }
        for (int q = worst; q < 4; ++q) list[q] = list[q + 1];
        cnt = 4;
      }
    }
  }
  if (lane == 0) {
    for (int q = 0; q < 4; ++q) nbr[4 * a + q] = q < cnt ? list[q] : -1;
    nbc[a] = cnt;
  }
}
__global__ void k_hbonds(int n, const int *__restrict__ z, const double *__restrict__ xyz, const int *__restrict__ nbr,
                         const int *__restrict__ nbc, double *__restrict__ e_out) {
  hbonds_warp(n, z, xyz, nbr, nbc, e_out, blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5));
}
__global__ void k_finish(int n_pairs_part, const double *__restrict__ pd, const double *__restrict__ py,
                         const double *__restrict__ ph, int n, const double *__restrict__ ehb,
                         const double *__restrict__ esioh, double *__restrict__ out) {
  finish_block(n_pairs_part, pd, py, ph, n, ehb, esioh, out);
}

// ---- batched: molecule = L.slot[blockIdx.z] (per-atom kernels) or a prefix item ----
__global__ void k_b_c6(BatchList L, const MolDesc *__restrict__ D) {
  const MolDesc &d = D[L.slot[blockIdx.z]];
  const CorrView v = corr_view(d.g.n_atoms, d.corr_scratch);
  c6_atom(v.n, d.g.z, d.g.xyz, d.smooth_dispersion, v.c6, blockIdx.x * blockDim.x + threadIdx.x);
}
__global__ void k_b_hb_neighbours(BatchList L, const MolDesc *__restrict__ D) {
  const MolDesc &d = D[L.slot[blockIdx.z]];
  const CorrView v = corr_view(d.g.n_atoms, d.corr_scratch);
  hb_neighbours_atom(v.n, d.g.z, d.g.xyz, v.nbr, v.nbc, blockIdx.x * blockDim.x + threadIdx.x);
}
__global__ void k_b_sioh(BatchList L, const MolDesc *__restrict__ D) {
  const MolDesc &d = D[L.slot[blockIdx.z]];
  const CorrView v = corr_view(d.g.n_atoms, d.corr_scratch);
  sioh_atom(v.n, d.g.z, d.g.xyz, v.esioh, blockIdx.x * blockDim.x + threadIdx.x);
}
__global__ void k_b_hbonds(BatchList L, const MolDesc *__restrict__ D) {
  const MolDesc &d = D[L.slot[blockIdx.z]];
  const CorrView v = corr_view(d.g.n_atoms, d.corr_scratch);
  hbonds_warp(v.n, d.g.z, d.g.xyz, v.nbr, v.nbc, v.ehb, blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5));
}
// item = (atom u, column block) of one molecule, as in the core-core sweep
__global__ void k_b_pair_corr(BatchList L, const MolDesc *__restrict__ D, int hh) {
  const int item = blockIdx.x;
  const int m = batch_find(L, item);
  const MolDesc &d = D[L.slot[m]];
  const CorrView v = corr_view(d.g.n_atoms, d.corr_scratch);
  const int local = item - L.prefix[m];
  const int u = local / v.gx, bx = local - u * v.gx;
  pair_corr_block(v.n, d.g.z, d.g.xyz, v.c6, hh, u, bx, (size_t)u * v.gx + bx, v.pd, v.py, v.ph);
}
__global__ void k_b_finish(BatchList L, const MolDesc *__restrict__ D, MolCtl *__restrict__ C, int zero) {
  const int slot = L.slot[blockIdx.x];
  const MolDesc &d = D[slot];
  if (zero) {
    if (threadIdx.x < 5) C[slot].corr[threadIdx.x] = 0.0;
    return;
  }
  const CorrView v = corr_view(d.g.n_atoms, d.corr_scratch);
  finish_block((int)v.parts, v.pd, v.py, v.ph, v.n, v.ehb, v.esioh, C[slot].corr);
}

// ---- gradient of the correction energy (src/gradient.rs:208-261) ----------------------
// Central differences (five-point, step kCorrStep) of the correction energy. With the
// default discrete C6 (bond counts, src/dispersion.rs:297-330: fixed under a small
// displacement, as the reference's gradient treats them) the pair terms (dispersion, C#C,
// PM7-HH) are differentiated pair by pair in r, and only the many-body H-bond and Si-O-H
// items are re-evaluated at displaced copies of the geometry -- and only those within reach
// of the moved atom, the others being bit-identical to the base values (covalent neighbour
// lists, a discrete choice, are taken at the base geometry). With the smooth C6
// (src/dispersion.rs:428-) every term is re-evaluated at every copy (plus one undisplaced
// copy for the base energy). The EH+ H-bond energy has jumps and kinks (the hard switches of
// hbond.rs:525-620), and in a large cluster some stencil always lands on one: the derivative
// is taken by robust_derivative (gradient.cuh), which falls back to the one-sided formula of
// the unbroken side -- the derivative of the branch the geometry is on, as the reference's
// analytic gradient gives it. The step is small (1e-5 Bohr) so that breaks are rarely inside
// a stencil; differencing only the changed items keeps the rounding error near 1e-12 kcal/mol.
constexpr double kCorrStep = 1.0e-5;  // Bohr
constexpr double kBreakTol = 1.0e-9;  // kcal/mol: third differences of a smooth term stay below it
constexpr double kSiohReachAng = 2.5;  // Si within 2.4 A, H within 1.4 A of the oxygen

// How far (Angstrom) the H-bond energies that depend on atom A reach, or -1 for none. The
// energy of hydrogen j (hbonds_warp) depends on j, its donors (N/O within 1.4 A), their
// acceptors (N/O within 7 A of the donor, so within 8.4 A of j) and the covalent neighbours of
// both (neighbour lists fixed at the base geometry). So A reaches 0 (itself, a hydrogen),
// 8.4 A (an N or O) and 8.4 A + |A - X| for each N/O atom X that lists A as a neighbour.
__global__ void k_hb_reach(int n, const int *__restrict__ z, const double *__restrict__ xyz,
                           const int *__restrict__ nbr, const int *__restrict__ nbc, double *__restrict__ reach) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= n) return;
  double r = z[a] == 1 ? 0.0 : -1.0;
  if (is_acceptor(z[a])) r = fmax(r, 8.4);
  for (int x = 0; x < n; ++x) {
    if (!is_acceptor(z[x])) continue;
    for (int q = 0; q < nbc[x]; ++q)
      if (nbr[4 * x + q] == a) r = fmax(r, 8.4 + dist_ang(xyz, x, a));
  }
  reach[a] = r;
}

// Copy c of a pass holds stencil point s = s0 + c: atom s / 12 moved by stencil_offset(s % 12);
// s = 12 n is the undisplaced geometry.
__global__ void k_fd_displace(int n, const double *__restrict__ xyz, int s0, size_t stride, double *__restrict__ work) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x, c = blockIdx.y;
  if (i >= 3 * n) return;
  const int s = s0 + c;
  double o[3] = {0.0, 0.0, 0.0};
  if (s < kStencil * n) stencil_offset(s % kStencil, kCorrStep, o);
  work[(size_t)c * stride + i] = xyz[i] + (i / 3 == s / kStencil ? o[i % 3] : 0.0);
}

// ... full path: the whole correction energy per copy (coordinates, corrections scratch, parts).
struct FdCopy {
  double *xyz;
  CorrView v;
  double *out;
};
__device__ __forceinline__ FdCopy fd_copy(int n, double *work, size_t stride, int c) {
  FdCopy f;
  f.xyz = work + (size_t)c * stride;
  f.v = corr_view(n, f.xyz + 3 * (size_t)n);
  const size_t parts = (size_t)((n + 127) / 128) * (size_t)(n > 0 ? n : 1);
  f.out = f.xyz + 3 * (size_t)n + 3 * parts + 11 * (size_t)n;
  return f;
}
__global__ void k_fd_c6(int n, const int *__restrict__ z, int smooth, double *work, size_t stride) {
  const FdCopy f = fd_copy(n, work, stride, blockIdx.z);
  c6_atom(n, z, f.xyz, smooth, f.v.c6, blockIdx.x * blockDim.x + threadIdx.x);
}
__global__ void k_fd_pair_corr(int n, const int *__restrict__ z, int hh, double *work, size_t stride) {
  const FdCopy f = fd_copy(n, work, stride, blockIdx.z);
  pair_corr_block(n, z, f.xyz, f.v.c6, hh, blockIdx.y, blockIdx.x, (size_t)blockIdx.y * gridDim.x + blockIdx.x,
                  f.v.pd, f.v.py, f.v.ph);
}
__global__ void k_fd_hb_neighbours(int n, const int *__restrict__ z, double *work, size_t stride) {
  const FdCopy f = fd_copy(n, work, stride, blockIdx.z);
  hb_neighbours_atom(n, z, f.xyz, f.v.nbr, f.v.nbc, blockIdx.x * blockDim.x + threadIdx.x);
}
__global__ void k_fd_hbonds(int n, const int *__restrict__ z, double *work, size_t stride) {
  const FdCopy f = fd_copy(n, work, stride, blockIdx.z);
  hbonds_warp(n, z, f.xyz, f.v.nbr, f.v.nbc, f.v.ehb, blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5));
}
__global__ void k_fd_sioh(int n, const int *__restrict__ z, double *work, size_t stride) {
  const FdCopy f = fd_copy(n, work, stride, blockIdx.z);
  sioh_atom(n, z, f.xyz, f.v.esioh, blockIdx.x * blockDim.x + threadIdx.x);
}
// The copy's total correction, summed in the order the result uses (scf.rs:907-932).
__global__ void k_fd_finish(int n, double *work, size_t stride, int s0, double *__restrict__ energies) {
  const FdCopy f = fd_copy(n, work, stride, blockIdx.x);
  finish_block((int)f.v.parts, f.v.pd, f.v.py, f.v.ph, n, f.v.ehb, f.v.esioh, f.out);
  if (threadIdx.x == 0) {
    double e = f.out[0];
    e += f.out[1];
    e += f.out[4];
    e += f.out[2];
    e += f.out[3];
    energies[s0 + blockIdx.x] = e;
  }
}

// ... local path: per copy, coordinates and the H-bond / Si-O-H energy of every atom.
struct FdLocal {
  double *xyz, *hb, *so;
};
__device__ __forceinline__ FdLocal fd_local(int n, double *work, size_t stride, int c) {
  FdLocal f;
  f.xyz = work + (size_t)c * stride;
  f.hb = f.xyz + 3 * (size_t)n;
  f.so = f.hb + n;
  return f;
}
// A warp per atom j of copy blockIdx.z: its H-bond energy, re-evaluated when j is a hydrogen
// within reach of the moved atom, else the base value.
__global__ void k_fd_hbonds_local(int n, const int *__restrict__ z, const int *__restrict__ nbr,
                                  const int *__restrict__ nbc, const double *__restrict__ ehb0,
                                  const double *__restrict__ reach, int s0, double *work, size_t stride) {
  const int j = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (j >= n) return;
  const FdLocal f = fd_local(n, work, stride, blockIdx.z);
  const int A = (s0 + (int)blockIdx.z) / kStencil;
  if (z[j] != 1 || reach[A] < 0.0 || dist_ang(f.xyz, j, A) > reach[A] + 0.01) {
    if ((threadIdx.x & 31) == 0) f.hb[j] = ehb0[j];
    return;
  }
  hbonds_warp(n, z, f.xyz, nbr, nbc, f.hb, j);
}
__global__ void k_fd_sioh_local(int n, const int *__restrict__ z, const double *__restrict__ esioh0, int s0, double *work,
                                size_t stride) {
  const int o = blockIdx.x * blockDim.x + threadIdx.x;
  if (o >= n) return;
  const FdLocal f = fd_local(n, work, stride, blockIdx.z);
  const int A = (s0 + (int)blockIdx.z) / kStencil;
  if (z[o] != 8 || dist_ang(f.xyz, o, A) > kSiohReachAng) f.so[o] = esioh0[o];
  else sioh_atom(n, z, f.xyz, f.so, o);
}
// ... H-bond terms by triple. The H-bond energy is a sum of eh_plus(donor i, hydrogen j,
// acceptor k) over the triples hbonds_warp selects; moving atom A changes only the triples
// whose evaluation reads A: i, j, k, the covalent neighbours of i and k and, for a side with a
// single neighbour y, the atoms bonded to y (assign_refs' second shell). The triples are
// selected once at the base geometry (a discrete choice, like the neighbour lists), each
// copy re-evaluates only its atom's triples, and the changes are summed.
constexpr int kHbDeps = 40;  // atoms a triple's value can depend on (3 + 4 + 4 + two shells)

__global__ void k_hb_tcount(int n, const int *__restrict__ z, const double *__restrict__ xyz, int *__restrict__ cnt) {
  const int j = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (j >= n) return;
  int c = 0;
  if (z[j] == 1) {
    for (int base = 0; base < n; base += 32) {
      const int i = base + lane;
      const bool donor = i < n && is_acceptor(z[i]) && dist2_ang(xyz, i, j) < 1.4 * 1.4;
      unsigned m = __ballot_sync(0xffffffffu, donor);
      while (m) {
        const int di = base + __ffs(m) - 1;
        m &= m - 1;
        for (int k = lane; k < n; k += 32) c += hb_acceptor_ok(z, xyz, j, di, k) ? 1 : 0;
      }
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
  if (lane == 0) cnt[j] = c;
}

// The triples of hydrogen j from position off[j] on (donor order, then acceptor order), with
// their base-geometry values.
__global__ void k_hb_tfill(int n, const int *__restrict__ z, const double *__restrict__ xyz,
                           const int *__restrict__ nbr, const int *__restrict__ nbc, const int *__restrict__ off,
                           int4 *__restrict__ tri, double *__restrict__ e0) {
  const int j = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (j >= n || z[j] != 1) return;
  int pos = off[j];
  for (int base = 0; base < n; base += 32) {
    const int i = base + lane;
    const bool donor = i < n && is_acceptor(z[i]) && dist2_ang(xyz, i, j) < 1.4 * 1.4;
    unsigned m = __ballot_sync(0xffffffffu, donor);
    while (m) {
      const int di = base + __ffs(m) - 1;
      m &= m - 1;
      for (int kb = 0; kb < n; kb += 32) {
        const int k = kb + lane;
        const bool sel = k < n && hb_acceptor_ok(z, xyz, j, di, k);
        const unsigned b = __ballot_sync(0xffffffffu, sel);
        if (sel) {
          const int t = pos + __popc(b & ((1u << lane) - 1u));
          tri[t] = make_int4(di, j, k, 0);
          e0[t] = eh_plus(n, z, xyz, nbr, nbc, di, j, k);
        }
        pos += __popc(b);
      }
    }
  }
}

__device__ __forceinline__ int add_dep(int *d, int c, int a) {
  for (int q = 0; q < c && q < kHbDeps; ++q)
    if (d[q] == a) return c;
  if (c < kHbDeps) d[c] = a;
  return c + 1;
}

// The atoms triple t's value reads (bonding test with a 0.05 A margin for the second shell).
__global__ void k_hb_tdeps(int T, int n, const int *__restrict__ z, const double *__restrict__ xyz,
                           const int *__restrict__ nbr, const int *__restrict__ nbc, const int4 *__restrict__ tri,
                           int *__restrict__ deps, int *__restrict__ overflow) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= T) return;
  const int4 q = tri[t];
  int d[kHbDeps];
  int c = 0;
  c = add_dep(d, c, q.x);
  c = add_dep(d, c, q.y);
  c = add_dep(d, c, q.z);
  const int side[2] = {q.x, q.z};
  for (int sd = 0; sd < 2; ++sd) {
    const int x = side[sd];
    for (int p = 0; p < nbc[x]; ++p) c = add_dep(d, c, nbr[4 * x + p]);
    if (nbc[x] == 1) {
      const int y = nbr[4 * x];
      for (int a = 0; a < n; ++a)
        if (a != y && dist_ang(xyz, a, y) < bonding(z, a, y) + 0.05) c = add_dep(d, c, a);
    }
  }
  if (c > kHbDeps) atomicOr(overflow, 1);
  for (int p = 0; p < kHbDeps; ++p) deps[(size_t)t * kHbDeps + p] = p < c && p < kHbDeps ? d[p] : -1;
}

// A warp per copy: the change of the H-bond energy, summed over the moved atom's triples.
__global__ void k_fd_hb_triples(int n, const int *__restrict__ z, const int *__restrict__ nbr,
                                const int *__restrict__ nbc, const int4 *__restrict__ tri,
                                const double *__restrict__ e0, const int *__restrict__ list_off,
                                const int *__restrict__ list, int s0, int copies, double *work, size_t stride,
                                double *__restrict__ energies) {
  const int c = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (c >= copies) return;
  const int s = s0 + c, A = s / kStencil;
  const double *X = work + (size_t)c * stride;
  double e = 0.0;
  for (int p = list_off[A] + lane; p < list_off[A + 1]; p += 32) {
    const int t = list[p];
    const int4 q = tri[t];
    e += eh_plus(n, z, X, nbr, nbc, q.x, q.y, q.z) - e0[t];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(0xffffffffu, e, o);
  if (lane == 0) energies[s] = e;
}

// The copy's change of the H-bond energy from whole-hydrogen re-evaluation (k_fd_hbonds_local).
__global__ void k_fd_finish_hb(int n, const double *__restrict__ ehb0, double *work, size_t stride, int s0,
                               double *__restrict__ energies) {
  const FdLocal f = fd_local(n, work, stride, blockIdx.x);
  double d = 0.0;
  for (int i = threadIdx.x; i < n; i += 256) d += f.hb[i] - ehb0[i];
  d = block_sum<256>(d);
  if (threadIdx.x == 0) energies[s0 + blockIdx.x] = d;
}

// Adds the copy's change of the Si-O-H energy.
__global__ void k_fd_finish_sioh(int n, const double *__restrict__ esioh0, double *work, size_t stride, int s0,
                                 double *__restrict__ energies) {
  const FdLocal f = fd_local(n, work, stride, blockIdx.x);
  double d = 0.0;
  for (int i = threadIdx.x; i < n; i += 256) d += f.so[i] - esioh0[i];
  d = block_sum<256>(d);
  if (threadIdx.x == 0) energies[s0 + blockIdx.x] += d;
}

// A warp per atom A: the pair terms' derivative along every pair (A, B) at fixed C6, by
// differences in r (robust_derivative: the PM7-HH term is piecewise); lanes over partners,
// fixed xor tree. kcal/mol per Bohr.
__global__ void k_corr_pair_grad(int n, const int *__restrict__ z, const double *__restrict__ xyz,
                                 const double *__restrict__ c6, int hh, double *__restrict__ grad) {
  const int A = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (A >= n) return;
  double acc[3] = {0.0, 0.0, 0.0};
  for (int B = lane; B < n; B += 32) {
    if (B == A) continue;
    const int u = A < B ? A : B, v = A < B ? B : A;
    const double d[3] = {xyz[3 * A] - xyz[3 * B], xyz[3 * A + 1] - xyz[3 * B + 1], xyz[3 * A + 2] - xyz[3 * B + 2]};
    const double r = sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    double e5[5];  // r - 2h .. r + 2h
    for (int q = 0; q < 5; ++q) {
      double ed, ey, eh;
      pair_corr_r(z[u], z[v], c6[u], c6[v], hh, r + (q - 2) * kCorrStep, ed, ey, eh);
      e5[q] = ed + 12.0 * ey + eh;
    }
    const double dedr = robust_derivative(e5[0], e5[1], e5[2], e5[3], e5[4], kCorrStep, kBreakTol);
    for (int k = 0; k < 3; ++k) acc[k] += dedr * (d[k] / r);
  }
  for (int k = 0; k < 3; ++k) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], o);
  }
  if (lane == 0)
    for (int k = 0; k < 3; ++k) grad[3 * A + k] = acc[k];
}

// energies[12 a + 4 k + j]: atom a moved along axis k by +h, -h, +2h, -2h (j = 0..3); the
// base energy is energies[12 n] (zero on the local path, which holds changes).
__global__ void k_fd_grad(int n, const double *__restrict__ energies, int add, double *__restrict__ grad) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= 3 * n) return;
  const double *e = energies + (size_t)(i / 3) * kStencil + 4 * (i % 3);
  const double g = robust_derivative(e[3], e[1], energies[(size_t)kStencil * n], e[0], e[2], kCorrStep, kBreakTol);
  grad[i] = add ? grad[i] + g : g;
}

// Work layout: a base block (the local path's C6, base H-bond and Si-O-H energies, reach,
// neighbour lists) then `copies` slices of `corr_copy_stride` doubles.
size_t corr_base_doubles(int n) { return 9 * (size_t)n + 8; }
size_t corr_copy_stride(int n, int smooth) {
  return smooth ? 3 * (size_t)n + corrections_scratch(n) + 8 : 5 * (size_t)n + 8;
}

}  // namespace

// Temporary device buffers of one call, freed on the stream however the call ends.
struct StreamTemps {
  cudaStream_t st;
  std::vector<void *> ptrs;
  explicit StreamTemps(cudaStream_t s) : st(s) {}
  StreamTemps(const StreamTemps &) = delete;
  StreamTemps &operator=(const StreamTemps &) = delete;
  template <class T>
  T *alloc(size_t count) {
    void *p = nullptr;
    CUDA_OK(cudaMallocAsync(&p, sizeof(T) * (count > 0 ? count : 1), st));
    ptrs.push_back(p);
    return static_cast<T *>(p);
  }
  ~StreamTemps() {
    for (void *p : ptrs) cudaFreeAsync(p, st);
  }
};

size_t corrections_gradient_work(int n_atoms, int copies, int smooth) {
  return corr_base_doubles(n_atoms) + (size_t)copies * corr_copy_stride(n_atoms, smooth);
}

void launch_corrections_gradient(cudaStream_t st, int n, const int *z, const double *xyz, int method, int smooth,
                                 int any_si, int copies, double *work, double *energies, double *grad) {
  if (n <= 0) return;
  if (method == 3) {  // PM7-minus carries no post-SCF corrections
    CUDA_OK(cudaMemsetAsync(grad, 0, 3 * sizeof(double) * (size_t)n, st));
    return;
  }
  const int hh = method == 4;
  const size_t stride = corr_copy_stride(n, smooth);
  double *base = work, *copy0 = work + corr_base_doubles(n);
  const int total = kStencil * n;
  const int ga = (n + 127) / 128;
  if (smooth) {
    for (int s0 = 0; s0 <= total; s0 += copies) {  // s = total: the base geometry
      const int c = copies < total + 1 - s0 ? copies : total + 1 - s0;
      k_fd_displace<<<dim3((3 * n + 127) / 128, c), 128, 0, st>>>(n, xyz, s0, stride, copy0);
      k_fd_c6<<<dim3(ga, 1, c), 128, 0, st>>>(n, z, smooth, copy0, stride);
      k_fd_pair_corr<<<dim3(ga, n, c), 128, 0, st>>>(n, z, hh, copy0, stride);
      k_fd_hb_neighbours<<<dim3(ga, 1, c), 128, 0, st>>>(n, z, copy0, stride);
      k_fd_hbonds<<<dim3((n + 3) / 4, 1, c), 128, 0, st>>>(n, z, copy0, stride);
      k_fd_sioh<<<dim3(ga, 1, c), 128, 0, st>>>(n, z, copy0, stride);
      k_fd_finish<<<c, 256, 0, st>>>(n, copy0, stride, s0, energies);
      note_launch(7);
    }
    k_fd_grad<<<(3 * n + 127) / 128, 128, 0, st>>>(n, energies, 0, grad);
    note_launch();
    return;
  }
  // base quantities of the local path
  double *c6 = base, *ehb0 = c6 + n, *esioh0 = ehb0 + n, *reach = esioh0 + n;
  int *nbr = reinterpret_cast<int *>(reach + n), *nbc = nbr + 4 * n;
  k_c6_discrete_warp<<<(n + 3) / 4, 128, 0, st>>>(n, z, xyz, c6);
  k_hb_neighbours_warp<<<(n + 3) / 4, 128, 0, st>>>(n, z, xyz, nbr, nbc);
  if (any_si) k_sioh<<<ga, 128, 0, st>>>(n, z, xyz, esioh0);  // without Si the term is zero
  k_corr_pair_grad<<<(n + 3) / 4, 128, 0, st>>>(n, z, xyz, c6, hh, grad);
  CUDA_OK(cudaMemsetAsync(energies + total, 0, sizeof(double), st));  // the local path holds changes
  note_launch(any_si ? 4 : 3);
  // the H-bond triples at the base geometry, their dependency atoms, and each atom's triples
  std::vector<int> cnt(n), off(n + 1, 0);
  StreamTemps tmp(st);
  int *d_cnt = tmp.alloc<int>(n + 1);
  k_hb_tcount<<<(n + 3) / 4, 128, 0, st>>>(n, z, xyz, d_cnt);
  note_launch();
  CUDA_OK(cudaMemcpyAsync(cnt.data(), d_cnt, sizeof(int) * n, cudaMemcpyDeviceToHost, st));
  CUDA_OK(cudaStreamSynchronize(st));
  for (int j = 0; j < n; ++j) off[j + 1] = off[j] + cnt[j];
  const int T = off[n];
  int4 *d_tri = nullptr;
  double *d_e0 = nullptr;
  int *d_deps = nullptr, *d_flag = nullptr, *d_list_off = nullptr, *d_list = nullptr;
  bool by_triple = true;
  if (T > 0) {
    d_tri = tmp.alloc<int4>(T);
    d_e0 = tmp.alloc<double>(T);
    d_deps = tmp.alloc<int>((size_t)T * kHbDeps);
    d_flag = tmp.alloc<int>(1);
    CUDA_OK(cudaMemsetAsync(d_flag, 0, sizeof(int), st));
    CUDA_OK(cudaMemcpyAsync(d_cnt, off.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice, st));
    k_hb_tfill<<<(n + 3) / 4, 128, 0, st>>>(n, z, xyz, nbr, nbc, d_cnt, d_tri, d_e0);
    k_hb_tdeps<<<(T + 127) / 128, 128, 0, st>>>(T, n, z, xyz, nbr, nbc, d_tri, d_deps, d_flag);
    note_launch(2);
    std::vector<int> deps((size_t)T * kHbDeps);
    int flag = 0;
    CUDA_OK(cudaMemcpyAsync(deps.data(), d_deps, sizeof(int) * deps.size(), cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaMemcpyAsync(&flag, d_flag, sizeof(int), cudaMemcpyDeviceToHost, st));
    CUDA_OK(cudaStreamSynchronize(st));
    by_triple = flag == 0;
    if (!by_triple) {  // the fallback's inputs: base H-bond energy per hydrogen, each atom's reach
      k_hbonds<<<(n + 3) / 4, 128, 0, st>>>(n, z, xyz, nbr, nbc, ehb0);
      k_hb_reach<<<ga, 128, 0, st>>>(n, z, xyz, nbr, nbc, reach);
      note_launch(2);
    } else {
      std::vector<int> loff(n + 1, 0), list;
      for (size_t q = 0; q < deps.size(); ++q)
        if (deps[q] >= 0) ++loff[deps[q] + 1];
      for (int a = 0; a < n; ++a) loff[a + 1] += loff[a];
      list.resize(loff[n]);
      std::vector<int> fill(loff.begin(), loff.end() - 1);
      for (int t = 0; t < T; ++t)  // ascending t within every atom's list
        for (int p = 0; p < kHbDeps; ++p) {
          const int a = deps[(size_t)t * kHbDeps + p];
          if (a >= 0) list[fill[a]++] = t;
        }
      d_list_off = tmp.alloc<int>(n + 1);
      d_list = tmp.alloc<int>(list.size());
      CUDA_OK(cudaMemcpyAsync(d_list_off, loff.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice, st));
      if (!list.empty())
        CUDA_OK(cudaMemcpyAsync(d_list, list.data(), sizeof(int) * list.size(), cudaMemcpyHostToDevice, st));
      CUDA_OK(cudaStreamSynchronize(st));  // the host vectors are about to go
    }
  }
  for (int s0 = 0; s0 < total; s0 += copies) {
    const int c = copies < total - s0 ? copies : total - s0;
    k_fd_displace<<<dim3((3 * n + 127) / 128, c), 128, 0, st>>>(n, xyz, s0, stride, copy0);
    if (T == 0) {
      CUDA_OK(cudaMemsetAsync(energies + s0, 0, sizeof(double) * c, st));
    } else if (by_triple) {
      k_fd_hb_triples<<<(c + 3) / 4, 128, 0, st>>>(n, z, nbr, nbc, d_tri, d_e0, d_list_off, d_list, s0, c, copy0, stride,
                                                   energies);
    } else {  // a triple reads more atoms than kept: re-evaluate every hydrogen within reach
      k_fd_hbonds_local<<<dim3((n + 3) / 4, 1, c), 128, 0, st>>>(n, z, nbr, nbc, ehb0, reach, s0, copy0, stride);
      k_fd_finish_hb<<<c, 256, 0, st>>>(n, ehb0, copy0, stride, s0, energies);
      note_launch();
    }
    if (any_si) {
      k_fd_sioh_local<<<dim3(ga, 1, c), 128, 0, st>>>(n, z, esioh0, s0, copy0, stride);
      k_fd_finish_sioh<<<c, 256, 0, st>>>(n, esioh0, copy0, stride, s0, energies);
      note_launch(2);
    }
    note_launch(T > 0 && by_triple ? 2 : 1);
  }
  CUDA_OK(cudaGetLastError());
  k_fd_grad<<<(3 * n + 127) / 128, 128, 0, st>>>(n, energies, 1, grad);
  note_launch();
}

size_t corrections_scratch(int n_atoms) {
  const size_t parts = (size_t)((n_atoms + 127) / 128) * (size_t)(n_atoms > 0 ? n_atoms : 1);
  return 3 * parts + 3 * (size_t)n_atoms + 8 * (size_t)n_atoms;
}

void launch_b_corrections(cudaStream_t st, const BatchList &Lmol, const BatchList &Lpairs, const MolDesc *D, MolCtl *C,
                          int method, int max_atoms) {
  if (Lmol.n <= 0) return;
  if (method == 3 || max_atoms == 0) {  // PM7-minus carries no post-SCF corrections
    k_b_finish<<<Lmol.n, 256, 0, st>>>(Lmol, D, C, 1);
    note_launch();
    return;
  }
  const int ga = (max_atoms + 127) / 128;
  k_b_c6<<<dim3(ga, 1, Lmol.n), 128, 0, st>>>(Lmol, D);
  if (Lpairs.total > 0) k_b_pair_corr<<<Lpairs.total, 128, 0, st>>>(Lpairs, D, method == 4);
  k_b_hb_neighbours<<<dim3(ga, 1, Lmol.n), 128, 0, st>>>(Lmol, D);
  k_b_hbonds<<<dim3((max_atoms + 3) / 4, 1, Lmol.n), 128, 0, st>>>(Lmol, D);
  k_b_sioh<<<dim3(ga, 1, Lmol.n), 128, 0, st>>>(Lmol, D);
  k_b_finish<<<Lmol.n, 256, 0, st>>>(Lmol, D, C, 0);
  note_launch(6);
}

void launch_corrections(cudaStream_t st, int n, const int *z, const double *xyz, int method, int smooth,
                        double *scratch, size_t, double *out) {
  if (method == 3 || n == 0) {  // PM7-minus carries no post-SCF corrections
    cudaMemsetAsync(out, 0, 5 * sizeof(double), st);
    return;
  }
  const int gx = (n + 127) / 128;
  const size_t parts = (size_t)gx * n;
  double *pd = scratch, *py = pd + parts, *ph = py + parts, *c6 = ph + parts, *ehb = c6 + n, *esioh = ehb + n;
  int *nbr = reinterpret_cast<int *>(esioh + n);
  int *nbc = nbr + 4 * n;
  if (smooth) k_c6<<<(n + 127) / 128, 128, 0, st>>>(n, z, xyz, smooth, c6);
  else k_c6_discrete_warp<<<(n + 3) / 4, 128, 0, st>>>(n, z, xyz, c6);
  note_launch();
  k_pair_corr<<<dim3(gx, n), 128, 0, st>>>(n, z, xyz, c6, method == 4, pd, py, ph);
  note_launch();
  k_hb_neighbours_warp<<<(n + 3) / 4, 128, 0, st>>>(n, z, xyz, nbr, nbc);
  note_launch();
  k_hbonds<<<(n + 3) / 4, 128, 0, st>>>(n, z, xyz, nbr, nbc, ehb);
  note_launch();
  k_sioh<<<(n + 127) / 128, 128, 0, st>>>(n, z, xyz, esioh);
  note_launch();
  k_finish<<<1, 256, 0, st>>>((int)parts, pd, py, ph, n, ehb, esioh, out);
  note_launch();
}

}  // namespace pm7
