// tri_face.cuh -- the per-face augmented Roe solver of TRITON, as a device
// function shared by every step kernel in this library.
//
// Reference: kernels_flux.h:84-273 (x faces, normal (1,0)) and :367-556
// (y faces, normal (0,1)).  "1" is the cell that owns the face, "2" the
// neighbour across it (east for x faces, NORTH for y faces: row-1).
//
// Bit-exactness contract: with T=double and the library's compile flags
// (--fmad=false, IEEE div/sqrt), every output equals the reference's bit for
// bit for finite states: each non-zero term keeps the reference's operand
// order and association.  Terms that are zero by construction are left out
// (products with the zero component of the face normal, contributions of a
// wave with zero speed, entropy-fix parts of waves without a fix): adding a
// zero never changes a non-zero sum, and a sum that is zero is flushed to +0
// before it is used, so only the sign of zeros inside the solver differs, and
// NaN propagation in a state that is already non-finite.
#pragma once

#include "tri_common.cuh"

namespace tri {

// Cell quantities every face of a cell uses, computed once per cell:
// velocities are zero below hextra (kernels_flux.h:98-117) and sqrt(h) is the
// reference's SQRTH array (kernels.h:178).
// z is the bed level (FP64 form) or the cell's FP32 offset from zb, the FP64
// base level of its 32x32 tile (FP32 form; zb is unused in FP64).
template <typename T>
struct CellQ {
  T h, qx, qy, z, sq, u, v;
  double zb;
};

template <typename T>
__device__ __forceinline__ CellQ<T> make_cell(T h, T qx, T qy, T z, T hextra, double zb = 0.0) {
  CellQ<T> c;
  c.h = h;
  c.qx = qx;
  c.qy = qy;
  c.z = z;
  c.zb = zb;
  c.sq = dev_fmax(dev_sqrt(h), T(0));
  if (h >= hextra) {
    const T rh = recip(h);
    c.u = div_shared(qx, h, rh);
    c.v = div_shared(qy, h, rh);
  } else {
    c.u = T(0);
    c.v = T(0);
  }
  return c;
}

// Result of one face: contributions to the owner (a) and to the neighbour (b),
// already scaled as rhs = dt*d/dx (kernels_flux.h:267-273).  'wet' is false for
// a dry-dry face (both scaled triples are then +0).
template <typename T>
struct FaceOut {
  T a0, a1, a2, b0, b1, b2;
};

// Step constants of the face solver: rdx = RN(1/dx) and rdt = RN(1/dt) turn
// the divisions by dx and dt into exact three-operation quotients.
template <typename T>
struct StepK {
  T dx, dt, rdx, rdt, hextra;
  bool dx_pow2;  // dx is a power of two: a / dx == a * rdx exactly (both round the same real)
};

// True for a positive normal power of two.
__host__ __device__ inline bool is_pow2(double x) {
  unsigned long long b;
#ifdef __CUDA_ARCH__
  b = (unsigned long long)__double_as_longlong(x);
#else
  __builtin_memcpy(&b, &x, 8);
#endif
  const unsigned long long e = b >> 52;
  return (b & 0x000FFFFFFFFFFFFFull) == 0 && e >= 1 && e <= 0x7FE;
}

template <typename T>
__host__ __device__ inline StepK<T> step_k(T dx, T dt, T rdx, T rdt, T hextra) {
  StepK<T> K;
  K.dx = dx;
  K.dt = dt;
  K.rdx = rdx;
  K.rdt = rdt;
  K.hextra = hextra;
  K.dx_pow2 = is_pow2((double)dx);
  return K;
}

// Products with the face normal (nx, ny) = (1,0) or (0,1): the component
// itself (the product with the zero component is a zero term).
template <typename T, bool XFACE>
__device__ __forceinline__ T n_dot(T a, T b) {  // a*nx + b*ny
  return XFACE ? a : b;
}
template <typename T, bool XFACE>
__device__ __forceinline__ T n_cross(T a, T b) {  // b*nx - a*ny
  return XFACE ? b : -a;
}

template <typename T, bool XFACE>
__device__ __forceinline__ FaceOut<T> face_flux(const CellQ<T>& c1, const CellQ<T>& c2, const StepK<T>& K) {
  const T dx = K.dx, dt = K.dt, hextra = K.hextra;
  const T G = T(kGravity), SG = T(kSqrtG), E12 = eps12<T>();
  FaceOut<T> out;
  out.a0 = out.a1 = out.a2 = out.b0 = out.b1 = out.b2 = T(0);

  const T h1 = c1.h, h2 = c2.h;
  if (!(h1 > T(0) || h2 > T(0))) return out;

  const T u1 = c1.u, v1 = c1.v, u2 = c2.u, v2 = c2.v;
  const T sqh1 = c1.sq, sqh2 = c2.sq;

  // Roe-averaged state and wave speeds
  const T h12 = T(0.5) * (h1 + h2);
  const T dh = h2 - h1;
  const T c12 = dev_sqrt(G * h12);
  const T rc12 = recip(c12);  // shared divisors: exact quotients via div_shared
  const T ssq = sqh1 + sqh2;
  const T rssq = recip(ssq);
  const T u12 = div_shared(u1 * sqh1 + u2 * sqh2, ssq, rssq);
  const T v12 = div_shared(v1 * sqh1 + v2 * sqh2, ssq, rssq);
  const T un = n_dot<T, XFACE>(u12, v12);
  T lam0 = un - c12, lam1 = un, lam2 = un + c12;
  T lamE0 = T(0), lamE2 = T(0);  // lamE1 is always zero

  // Harten-Hyman style entropy fix on the acoustic waves
  {
    const T un1 = n_dot<T, XFACE>(u1, v1), un2 = n_dot<T, XFACE>(u2, v2);
    T e1 = un1 - SG * sqh1;
    T e2 = un2 - SG * sqh2;
    if (e1 < T(0) && e2 > T(0)) {
      const T t = div_rare(e1 * (e2 - lam0), e2 - e1);
      lamE0 = lam0 - t;
      lam0 = t;
    }
    e1 = un1 + SG * sqh1;
    e2 = un2 + SG * sqh2;
    if (e1 < T(0) && e2 > T(0)) {
      const T t = div_rare(e2 * (lam2 - e1), e2 - e1);
      lamE2 = lam2 - t;
      lam2 = t;
    }
  }

  // eigenvector components (row 0 and row 2 have a leading 1, row 1 a 0)
  // (components that are zero for this face direction are never used)
  const T r01 = XFACE ? u12 - c12 : u12, r02 = XFACE ? v12 : v12 - c12;
  const T r11 = -c12, r12 = c12;  // wave 1: (0, -c12*ny, c12*nx)
  const T r21 = XFACE ? u12 + c12 : u12, r22 = XFACE ? v12 : v12 + c12;

  // wave strengths
  const T dqx = c2.qx - c1.qx, dqy = c2.qy - c1.qy;
  const T aq = div_shared(n_dot<T, XFACE>(dqx, dqy) - un * dh, c12, rc12);
  const T al0 = T(0.5) * (dh - aq);
  const T al1 = div_shared(n_cross<T, XFACE>(dqx - u12 * dh, dqy - v12 * dh), c12, rc12);
  const T al2 = T(0.5) * (dh + aq);

  // upwinded bed-step source, limited where the step is higher than the water
  T dz;
  bool above1, above2;  // z1 + h1 < z2, z2 + h2 < z1
  if (sizeof(T) == 8) {
    const T z1 = c1.z, z2 = c2.z;
    dz = z2 - z1;
    above1 = z1 + h1 < z2;
    above2 = z2 + h2 < z1;
  } else {
    // FP32 form: the bed step from each cell's own (base, offset) pair, so
    // every evaluation of a face gets the same value (a face on a tile edge
    // is evaluated by both tiles, and mass is conserved only if both agree)
    dz = c1.zb == c2.zb ? c2.z - c1.z : (T)((c2.zb - c1.zb) + ((double)c2.z - (double)c1.z));
    above1 = h1 < dz;
    above2 = h2 < -dz;
  }
  T dzp = dz, hp;
  if (dz >= T(0)) {
    hp = h1;
    if (above1) dzp = h1;
  } else {
    hp = h2;
    if (above2) dzp = -h2;
  }
  T be0 = div_shared(T(0.5) * G * (hp - T(0.5) * dev_fabs(dzp)) * dzp, c12, rc12);

  // positivity limiter on subcritical wet-wet faces
  hp = h1 + al0;
  if (lam0 * lam2 < T(0) && hp > T(0) && h1 > T(0) && h2 > T(0)) {
    // lam/(lam + lamE) is exactly 1 without an entropy-fix part (lam != 0 here)
    const T f0 = lamE2 == T(0) ? T(1) : div_rare(lam0, lam0 + lamE2);
    const T f2 = lamE0 == T(0) ? T(1) : div_rare(lam2, lam2 + lamE0);
    be0 = dev_fmax(be0, f0 * (al0 * lam0 - div_nz(h1 * dx * T(0.5), dt, K.rdt) + lamE2 * h2));
    be0 = dev_fmin(be0, f2 * (-al2 * lam2 + div_nz(h2 * dx * T(0.5), dt, K.rdt) + lamE0 * h1));
  }
  const T be2 = -be0;
  const T be1 = T(0);

  // intermediate states decide whether mass is redirected from a dry side;
  // they only matter next to a dry cell, so they are formed only there
  T p0 = T(0), p1 = T(0), p2 = T(0);  // owner side
  T q0 = T(0), q1 = T(0), q2 = T(0);  // neighbour side
  if (h2 < E12 && hp + div_rare(be2, lam2) < -E12) {
    p0 += (lam0 * al0 - be0) + (lam2 * al2 - be2);
  } else if (h1 < E12 && hp - div_rare(be0, lam0) < -E12) {
    q0 += (lam0 * al0 - be0) + (lam2 * al2 - be2);
  } else {
    // wave 0: eigenvector (1, r01, r02)
    {
      const T w = lam0 * al0 - be0;
      if (lam0 > T(0)) {
        q0 += w * T(1);
        q1 += w * r01;
        q2 += w * r02;
      } else {
        p0 += w * T(1);
        p1 += w * r01;
        p2 += w * r02;
      }
    }
    // wave 1: eigenvector (0, r11, r12)
    {
      const T w = lam1 * al1 - be1;
      if (lam1 > T(0)) {
        if (XFACE) q2 += w * r12; else q1 += w * r11;
      } else {
        if (XFACE) p2 += w * r12; else p1 += w * r11;
      }
    }
    // wave 2: eigenvector (1, r21, r22)
    {
      const T w = lam2 * al2 - be2;
      if (lam2 > T(0)) {
        q0 += w * T(1);
        q1 += w * r21;
        q2 += w * r22;
      } else {
        p0 += w * T(1);
        p1 += w * r21;
        p2 += w * r22;
      }
    }
  }
  // entropy-fix parts (a wave without a fix contributes zeros; lamE1 is zero)
  if (lamE0 != T(0)) {
    const T w = lamE0 * al0;
    if (lamE0 > T(0)) {
      q0 += w * T(1);
      q1 += w * r01;
      q2 += w * r02;
    } else {
      p0 += w * T(1);
      p1 += w * r01;
      p2 += w * r02;
    }
  }
  if (lamE2 != T(0)) {
    const T w = lamE2 * al2;
    if (lamE2 > T(0)) {
      q0 += w * T(1);
      q1 += w * r21;
      q2 += w * r22;
    } else {
      p0 += w * T(1);
      p1 += w * r21;
      p2 += w * r22;
    }
  }
  // flush tiny contributions, then scale to depth/discharge increments
  T th0 = E12;
  const T th1 = E12;
  if (sizeof(T) == 4) {
    // FP32 form: a mass contribution within the rounding noise of the terms
    // that formed it is noise.  1e-12 lies far above FP64 noise but far below
    // FP32 noise: at a shoreline the fluctuation into a dry cell cancels to
    // FP32 noise (~1e-9), which would leave 1e-11 m of water there, make the
    // cell count as wet and let water climb the bank.  (Momentum
    // contributions keep the absolute threshold only: zeroing those below
    // the noise of their terms deleted slow flows out of deep water every
    // step, and the FP32 run drained 2-5x further from FP64 in volume.)
    const T s0 = dev_fabs(lam0 * al0) + dev_fabs(be0) + dev_fabs(lam2 * al2) + dev_fabs(lamE0 * al0) +
                 dev_fabs(lamE2 * al2);
    th0 = dev_fmax(E12, T(kNoise32) * s0);
  }
  if (sizeof(T) == 4 && th0 > E12) {
    // FP32 form: a mass contribution that is noise moves to the other side
    // instead of vanishing, so the face still conserves mass; the dry side of
    // a shoreline face gets exactly nothing
    const bool np = dev_fabs(p0) < th0, nq = dev_fabs(q0) < th0;
    if (nq && (!np || h1 >= h2)) {  // both noise: to the side with more water
      p0 += q0;
      q0 = T(0);
    } else if (np) {
      q0 += p0;
      p0 = T(0);
    }
  }
  if (dev_fabs(p0) < E12) p0 = T(0);
  if (dev_fabs(q0) < E12) q0 = T(0);
  if (dev_fabs(p1) < th1) p1 = T(0);
  if (dev_fabs(q1) < th1) q1 = T(0);
  if (dev_fabs(p2) < th1) p2 = T(0);
  if (dev_fabs(q2) < th1) q2 = T(0);
  // rhs = dt*p/dx (kernels_flux.h:267-273); dt*p is +0 or at least dt*1e-12
  if (K.dx_pow2) {  // uniform over the launch
    const T s = K.rdx;
    out.a0 = (dt * p0) * s;
    out.a1 = (dt * p1) * s;
    out.a2 = (dt * p2) * s;
    out.b0 = (dt * q0) * s;
    out.b1 = (dt * q1) * s;
    out.b2 = (dt * q2) * s;
  } else {
    out.a0 = div_nz(dt * p0, dx, K.rdx);
    out.a1 = div_nz(dt * p1, dx, K.rdx);
    out.a2 = div_nz(dt * p2, dx, K.rdx);
    out.b0 = div_nz(dt * q0, dx, K.rdx);
    out.b1 = div_nz(dt * q1, dx, K.rdx);
    out.b2 = div_nz(dt * q2, dx, K.rdx);
  }
  return out;
}

}  // namespace tri
