// Forward-mode dual numbers with four tangents, and the P2G material map
// Phi: F* -> (F_out, tau) written once for float and for duals.  The adjoint
// kernels evaluate Phi on duals seeded with the four entries of F* to obtain
// the exact Jacobians of the branchy map the forward evaluates (taichi's 2x2
// SVD with its |S01| < 1e-5 and ordering branches, the 1e-6 singular-value
// floor, the payload's clamp to [1 - 5e-3, 1 + 5e-3], water's sqrt(J) I).
#pragma once
#include "jf_device.cuh"

struct D4 {
  float v;
  float d[4];
};

__device__ __forceinline__ D4 d4c(float v) { return D4{v, {0.f, 0.f, 0.f, 0.f}}; }
__device__ __forceinline__ D4 operator+(D4 a, D4 b) {
  return D4{a.v + b.v, {a.d[0] + b.d[0], a.d[1] + b.d[1], a.d[2] + b.d[2], a.d[3] + b.d[3]}};
}
__device__ __forceinline__ D4 operator-(D4 a, D4 b) {
  return D4{a.v - b.v, {a.d[0] - b.d[0], a.d[1] - b.d[1], a.d[2] - b.d[2], a.d[3] - b.d[3]}};
}
__device__ __forceinline__ D4 operator-(D4 a) { return D4{-a.v, {-a.d[0], -a.d[1], -a.d[2], -a.d[3]}}; }
__device__ __forceinline__ D4 operator*(D4 a, D4 b) {
  return D4{a.v * b.v, {a.d[0] * b.v + a.v * b.d[0], a.d[1] * b.v + a.v * b.d[1],
                        a.d[2] * b.v + a.v * b.d[2], a.d[3] * b.v + a.v * b.d[3]}};
}
__device__ __forceinline__ D4 operator*(float a, D4 b) {
  return D4{a * b.v, {a * b.d[0], a * b.d[1], a * b.d[2], a * b.d[3]}};
}
__device__ __forceinline__ D4 operator*(D4 a, float b) { return b * a; }
__device__ __forceinline__ D4 operator+(D4 a, float b) { return D4{a.v + b, {a.d[0], a.d[1], a.d[2], a.d[3]}}; }
__device__ __forceinline__ D4 operator+(float a, D4 b) { return b + a; }
__device__ __forceinline__ D4 operator-(D4 a, float b) { return D4{a.v - b, {a.d[0], a.d[1], a.d[2], a.d[3]}}; }
__device__ __forceinline__ D4 operator-(float a, D4 b) { return -(b - a); }
__device__ __forceinline__ D4 operator/(D4 a, D4 b) {
  const float q = a.v / b.v;
  const float ib = 1.0f / b.v;
  return D4{q, {(a.d[0] - q * b.d[0]) * ib, (a.d[1] - q * b.d[1]) * ib, (a.d[2] - q * b.d[2]) * ib,
                (a.d[3] - q * b.d[3]) * ib}};
}
__device__ __forceinline__ D4 operator/(float a, D4 b) { return d4c(a) / b; }
__device__ __forceinline__ D4 dsqrt(D4 a) {
  const float r = sqrtf(a.v);
  const float k = r > 0.0f ? 0.5f / r : 0.0f;
  return D4{r, {a.d[0] * k, a.d[1] * k, a.d[2] * k, a.d[3] * k}};
}
__device__ __forceinline__ float val(float a) { return a; }
__device__ __forceinline__ float val(D4 a) { return a.v; }
__device__ __forceinline__ float dsqrt(float a) { return sqrtf(a); }

// scalar constant in the type T
template <class T> __device__ __forceinline__ T tconst(float v);
template <> __device__ __forceinline__ float tconst<float>(float v) { return v; }
template <> __device__ __forceinline__ D4 tconst<D4>(float v) { return d4c(v); }

template <class T>
__device__ __forceinline__ T tmax(T a, float b) { return val(a) > b ? a : tconst<T>(b); }
template <class T>
__device__ __forceinline__ T tmin(T a, float b) { return val(a) < b ? a : tconst<T>(b); }
template <class T>
__device__ __forceinline__ T tabs(T a) { return val(a) < 0.0f ? -a : a; }

// Phi of the P2G material update (mpm_sim.py:206-233), for the adjoint.
// A = F* = (I + dt C) F row-major.  Outputs F_out (the stored deformation
// gradient), the Kirchhoff stress tau (without the dt * p_vol scaling) and
// J; the muscle's active term enters as pressure * J * d d^T.
template <class T>
__device__ __forceinline__ void jf_phi(const T A[4], int mt, float mu, float la, float pressure, float2 fd,
                                       T Fout[4], T tau[4], T& J) {
  const T x = A[0] + A[3];
  const T y = A[2] - A[1];
  const T scale = tconst<T>(1.0f) / dsqrt(x * x + y * y);
  const T c = x * scale, s = y * scale, ms = -s;
  const T S00 = c * A[0] + s * A[2];
  const T S01 = c * A[1] + s * A[3];
  const T S11 = ms * A[1] + c * A[3];
  T cc, ss, s1, s2;
  if (fabsf(val(S01)) < 1e-5f) {
    cc = tconst<T>(1.0f);
    ss = tconst<T>(0.0f);
    s1 = S00;
    s2 = S11;
  } else {
    const T tao = 0.5f * (S00 - S11);
    const T w = dsqrt(tao * tao + S01 * S01);
    const T t = val(tao) > 0.0f ? S01 / (tao + w) : S01 / (tao - w);
    cc = tconst<T>(1.0f) / dsqrt(t * t + 1.0f);
    ss = -t * cc;
    s1 = (cc * cc * S00 - 2.0f * cc * ss * S01) + ss * ss * S11;
    s2 = (ss * ss * S00 + 2.0f * cc * ss * S01) + cc * cc * S11;
  }
  T V00, V01, V10, V11;
  if (val(s1) < val(s2)) {
    const T tmp = s1;
    s1 = s2;
    s2 = tmp;
    V00 = -ss; V01 = cc; V10 = -cc; V11 = -ss;
  } else {
    V00 = cc; V01 = ss; V10 = -ss; V11 = cc;
  }
  const T U00 = c * V00 + ms * V10, U01 = c * V01 + ms * V11;
  const T U10 = s * V00 + c * V10, U11 = s * V01 + c * V11;
  s1 = tmax(s1, 1e-6f);
  s2 = tmax(s2, 1e-6f);
  if (mt == 2) {
    s1 = tmin(tmax(s1, 0.995f), 1.005f);
    s2 = tmin(tmax(s2, 0.995f), 1.005f);
  }
  J = s1 * s2;
  if (mt == 0) {
    const T sj = dsqrt(J);
    Fout[0] = sj; Fout[1] = tconst<T>(0.0f); Fout[2] = tconst<T>(0.0f); Fout[3] = sj;
  } else if (mt == 2) {
    const T a00 = U00 * s1, a01 = U01 * s2, a10 = U10 * s1, a11 = U11 * s2;
    Fout[0] = a00 * V00 + a01 * V01;
    Fout[1] = a00 * V10 + a01 * V11;
    Fout[2] = a10 * V00 + a11 * V01;
    Fout[3] = a10 * V10 + a11 * V11;
  } else {
    Fout[0] = A[0]; Fout[1] = A[1]; Fout[2] = A[2]; Fout[3] = A[3];
  }
  const T R00 = U00 * V00 + U01 * V01, R01 = U00 * V10 + U01 * V11;
  const T R10 = U10 * V00 + U11 * V01, R11 = U10 * V10 + U11 * V11;
  const float twomu = 2.0f * mu;
  const T E00 = twomu * (Fout[0] - R00), E01 = twomu * (Fout[1] - R01);
  const T E10 = twomu * (Fout[2] - R10), E11 = twomu * (Fout[3] - R11);
  const T diag = la * J * (J - 1.0f);
  tau[0] = (E00 * Fout[0] + E01 * Fout[1]) + diag;
  tau[1] = E00 * Fout[2] + E01 * Fout[3];
  tau[2] = E10 * Fout[0] + E11 * Fout[1];
  tau[3] = (E10 * Fout[2] + E11 * Fout[3]) + diag;
  if (mt == 3) {
    tau[0] = tau[0] + (fd.x * fd.x * pressure) * J;
    tau[1] = tau[1] + (fd.x * fd.y * pressure) * J;
    tau[2] = tau[2] + (fd.y * fd.x * pressure) * J;
    tau[3] = tau[3] + (fd.y * fd.y * pressure) * J;
  }
}
