// narrow.cuh -- FP64 narrow phase shared by the contact kernels and the
// fused LBVH queries: closest points of a vertex-triangle or edge-edge pair,
// the conservative time of impact of a moving pair, and the min-reduction of
// times of impact (exact in any order).
#pragma once

#include "common.cuh"

namespace ando {

// Segment-segment closest points (collision.cpp:389-452 scheme) with the
// segment parameters.
__device__ inline double ee_dist(d3 p0, d3 p1, d3 q0, d3 q1, double& s, double& t, d3& wp, d3& wq) {
  d3 d1 = p1 - p0, d2 = q1 - q0, r = p0 - q0;
  double a = dot(d1, d1), e = dot(d2, d2), f = dot(d2, r);
  const double eps = 1e-10;
  auto cl = [](double v) { return fmin(fmax(v, 0.0), 1.0); };
  s = 0.0; t = 0.0;
  if (a <= eps && e <= eps) { wp = p0; wq = q0; }
  else {
    if (a <= eps) { s = 0; t = cl(f / e); }
    else {
      double c = dot(d1, r);
      if (e <= eps) { t = 0; s = cl(-c / a); }
      else {
        double b = dot(d1, d2), den = a * e - b * b;
        s = den != 0.0 ? cl((b * f - c * e) / den) : 0.0;
        t = (b * s + f) / e;
        if (t < 0.0) { t = 0; s = cl(-c / a); }
        else if (t > 1.0) { t = 1; s = cl((b - c) / a); }
      }
    }
    wp = p0 + d1 * s; wq = q0 + d2 * t;
  }
  return nrm(wp - wq);
}

// Point-triangle distance (collision.cpp:279-386 scheme).
__device__ inline double pt_dist(d3 p, d3 a, d3 b, d3 c, d3& normal, d3& wq) {
  d3 ab = b - a, ac = c - a, ap = p - a;
  double d1 = dot(ab, ap), d2 = dot(ac, ap), dist;
  auto vert = [&](d3 q) { wq = q; d3 df = p - q; double dd = nrm(df); normal = dd > 1e-10 ? df / dd : mk(0, 0, 1); return dd; };
  if (d1 <= 0.0 && d2 <= 0.0) return vert(a);
  d3 bp = p - b; double d3_ = dot(ab, bp), d4 = dot(ac, bp);
  if (d3_ >= 0.0 && d4 <= d3_) return vert(b);
  d3 cp = p - c; double d5 = dot(ab, cp), d6 = dot(ac, cp);
  if (d6 >= 0.0 && d5 <= d6) return vert(c);
  double vc = d1 * d4 - d3_ * d2;
  if (vc <= 0.0 && d1 >= 0.0 && d3_ <= 0.0) return vert(a + ab * (d1 / (d1 - d3_)));
  double vb = d5 * d2 - d1 * d6;
  if (vb <= 0.0 && d2 >= 0.0 && d6 <= 0.0) return vert(a + ac * (d2 / (d2 - d6)));
  double va = d3_ * d6 - d5 * d4;
  if (va <= 0.0 && (d4 - d3_) >= 0.0 && (d5 - d6) >= 0.0) return vert(b + (c - b) * ((d4 - d3_) / ((d4 - d3_) + (d5 - d6))));
  double den = 1.0 / (va + vb + vc);
  wq = a + ab * (vb * den) + ac * (vc * den);
  d3 df = p - wq; dist = nrm(df);
  d3 tn = cross(ab, ac); double ta = nrm(tn);
  if (ta > 1e-10) { tn = tn / ta; if (dot(tn, df) < 0.0) tn = -tn; normal = tn; }
  else normal = dist > 1e-10 ? df / dist : mk(0, 0, 1);
  return dist;
}

__device__ inline void atomic_min_pos(unsigned long long* addr, double t) {
  atomicMin(addr, (unsigned long long)__double_as_longlong(fmax(t, 0.0)));
}
__device__ inline double warp_min(double v) { for (int o = 16; o; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o)); return v; }

// Conservative advancement: the distance of a pair cannot shrink faster than
// l (sum of the largest displacements of either side) per unit time, so
// stepping by (d - eta) / l never skips contact; stop at eta = d0 / 10. A
// pair that already touches (d0 = 0; only a kinematic pin snap can make one)
// cannot be advanced conservatively and does not bound the step: with it in,
// every later line search of the scene would return 0 and freeze the cloth.
// With eta_min > 0 (the kinematic pin pass) the move may not bring a pair
// closer than eta_min at all: pins that keep consuming 90% of a gap every
// frame would squeeze it to nothing, and no later line search could separate
// the pair.
//
// A pair closer than `near` at the start is where conservative advancement
// breaks down: it cannot tell a pair moving apart from one closing in, so it
// returns t ~ d0 / l and a pair squeezed to 1e-12 m would freeze every later
// line search. Such a pair is sampled instead (geometric times 2^-40..2^-1,
// then 0.5..1 in steps of 1/32): the step is allowed up to the last sample
// before the distance first falls below half its starting value.
template <class F> __device__ inline double advance(F dist, double l, double eta_min, double near) {
  if (!(l > 0.0)) return 1.0;
  double d0 = dist(0.0);
  if (!(d0 > 0.0)) return 1.0;
  if (d0 <= eta_min) return 0.0;
  if (d0 < near) {
    double prev = 0.0;
    for (int k = 40; k >= 1; --k) {
      double ts = ldexp(1.0, -k);
      if (!(dist(ts) >= 0.5 * d0)) return prev;
      prev = ts;
    }
    for (int k = 17; k <= 32; ++k) {
      double ts = double(k) / 32.0;
      if (!(dist(ts) >= 0.5 * d0)) return prev;
      prev = ts;
    }
    return 1.0;
  }
  double eta = fmax(0.1 * d0, eta_min), t = 0.0, d = d0;
  for (int it = 0; it < 200; ++it) {
    if (it) d = dist(t);
    if (d <= eta) return t;
    t += (d - eta) / l;
    if (t >= 1.0) return 1.0;
  }
  return t;
}

// Time of impact of pair (kind 0: vertex id[0] against triangle id[1..3];
// kind 1: edge id[0..1] against edge id[2..3]) moving x -> x + ext. The
// distance only depends on the relative motion of the four vertices, so the
// bound l on its rate of change is taken from the displacements minus their
// mean (additive CCD): two layers sliding together bound nothing, where the
// absolute displacements would cap the step at about 200 d0 / l.
__device__ inline double pair_toi(int kind, const int id[4], const double* x, const double* ext, double eta_min, double near) {
  d3 p[4], e[4];
  double L[4];
  for (int q = 0; q < 4; ++q) { p[q] = ld3(x, id[q]); e[q] = ld3(ext, id[q]); }
  const d3 mean = (e[0] + e[1] + e[2] + e[3]) * 0.25;
  for (int q = 0; q < 4; ++q) L[q] = nrm(e[q] - mean);
  if (kind == 0) {
    double l = L[0] + fmax(L[1], fmax(L[2], L[3]));
    return advance([&](double s) { d3 n, wq; return pt_dist(p[0] + e[0] * s, p[1] + e[1] * s, p[2] + e[2] * s, p[3] + e[3] * s, n, wq); }, l,
                   eta_min, near);
  }
  double l = fmax(L[0], L[1]) + fmax(L[2], L[3]);
  return advance([&](double s) { double a, b; d3 wp, wq; return ee_dist(p[0] + e[0] * s, p[1] + e[1] * s, p[2] + e[2] * s, p[3] + e[3] * s, a, b, wp, wq); },
                 l, eta_min, near);
}

// Distance of the pair at x (same closest-point schemes as the contacts).
__device__ inline double pair_gap(int kind, const int id[4], const double* x) {
  if (kind == 0) { d3 n, wq; return pt_dist(ld3(x, id[0]), ld3(x, id[1]), ld3(x, id[2]), ld3(x, id[3]), n, wq); }
  double s, t; d3 wp, wq;
  return ee_dist(ld3(x, id[0]), ld3(x, id[1]), ld3(x, id[2]), ld3(x, id[3]), s, t, wp, wq);
}

}  // namespace ando
