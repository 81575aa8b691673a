// epilogue.cuh -- per-vertex force assembly shared by every force kernel.
//
// Restates the tail of computeForceRange and computeSwingTractionRange
// (src/embedders/gvizForceEmbedder.c:117-124, 128-138) in FP64:
//   f = att + rep; |att|, |rep|; structForce = f;
//   disp = f - gravityK*(deg+1) * p/|p|   (skipped when |p| < 1e-9,
//          include/core/gvizVec.h:636-647; gravity uses the raw degree)
//   swing = m*|f - f_old|, traction = m*0.5*|f + f_old| on structForce.
#pragma once
#include "internal.cuh"

struct EpiArgs {
  const double2 *pos;
  const uint32_t *degree;
  const double *mass;
  double2 *sf;
  const double2 *sfOld;
  double2 *disp;
  double *att, *rep, *swing, *trac;
  double2 *repVec;  // optional: repulsion vectors (error measurements)
  double gravityK;
};

__device__ __forceinline__ void force_epilogue(const EpiArgs &e, uint32_t v,
                                               double ax, double ay, double rx,
                                               double ry) {
  double fx = 0.0, fy = 0.0;
  fx += ax;
  fy += ay;
  fx += rx;
  fy += ry;
  e.att[v] = sqrt(ax * ax + ay * ay);
  e.rep[v] = sqrt(rx * rx + ry * ry);
  if (e.repVec) e.repVec[v] = make_double2(rx, ry);
  e.sf[v] = make_double2(fx, fy);
  const double2 o = e.sfOld[v];
  const double m = e.mass[v];
  const double d0 = fx - o.x, d1 = fy - o.y;
  const double s0 = fx + o.x, s1 = fy + o.y;
  e.swing[v] = m * sqrt(d0 * d0 + d1 * d1);
  e.trac[v] = m * 0.5 * sqrt(s0 * s0 + s1 * s1);
  const double gmag = e.gravityK * (double)(e.degree[v] + 1u);
  const double2 p = e.pos[v];
  const double gd = sqrt(p.x * p.x + p.y * p.y);
  if (!(gd < 1e-9)) {
    const double s = gmag / gd;
    fx -= s * p.x;
    fy -= s * p.y;
  }
  e.disp[v] = make_double2(fx, fy);
}
