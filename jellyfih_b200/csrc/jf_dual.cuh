// Forward-mode dual numbers with four tangents, and the P2G material map
// Phi: F* -> (F_out, tau) written once for real numbers and for duals, in FP32
// and FP64 (R).  The adjoint kernels evaluate Phi on duals seeded with the four
// entries of F* to obtain the exact Jacobians of the branchy map the forward
// evaluates (taichi's 2x2 SVD with its |S01| < 1e-5 and ordering branches, the
// 1e-6 singular-value floor, the payload's clamp to [1 - 5e-3, 1 + 5e-3],
// water's sqrt(J) I).
#pragma once
#include "jf_device.cuh"

template <class R>
struct D4T {
  R v;
  R d[4];
};
using D4 = D4T<float>;

template <class R> __device__ __forceinline__ D4T<R> d4c(R v) { return D4T<R>{v, {R(0), R(0), R(0), R(0)}}; }
template <class R> __device__ __forceinline__ D4T<R> operator+(D4T<R> a, D4T<R> b) {
  return D4T<R>{a.v + b.v, {a.d[0] + b.d[0], a.d[1] + b.d[1], a.d[2] + b.d[2], a.d[3] + b.d[3]}};
}
template <class R> __device__ __forceinline__ D4T<R> operator-(D4T<R> a, D4T<R> b) {
  return D4T<R>{a.v - b.v, {a.d[0] - b.d[0], a.d[1] - b.d[1], a.d[2] - b.d[2], a.d[3] - b.d[3]}};
}
template <class R> __device__ __forceinline__ D4T<R> operator-(D4T<R> a) {
  return D4T<R>{-a.v, {-a.d[0], -a.d[1], -a.d[2], -a.d[3]}};
}
template <class R> __device__ __forceinline__ D4T<R> operator*(D4T<R> a, D4T<R> b) {
  return D4T<R>{a.v * b.v, {a.d[0] * b.v + a.v * b.d[0], a.d[1] * b.v + a.v * b.d[1],
                            a.d[2] * b.v + a.v * b.d[2], a.d[3] * b.v + a.v * b.d[3]}};
}
template <class R> __device__ __forceinline__ D4T<R> operator*(R a, D4T<R> b) {
  return D4T<R>{a * b.v, {a * b.d[0], a * b.d[1], a * b.d[2], a * b.d[3]}};
}
template <class R> __device__ __forceinline__ D4T<R> operator*(D4T<R> a, R b) { return b * a; }
template <class R> __device__ __forceinline__ D4T<R> operator+(D4T<R> a, R b) {
  return D4T<R>{a.v + b, {a.d[0], a.d[1], a.d[2], a.d[3]}};
}
template <class R> __device__ __forceinline__ D4T<R> operator+(R a, D4T<R> b) { return b + a; }
template <class R> __device__ __forceinline__ D4T<R> operator-(D4T<R> a, R b) {
  return D4T<R>{a.v - b, {a.d[0], a.d[1], a.d[2], a.d[3]}};
}
template <class R> __device__ __forceinline__ D4T<R> operator-(R a, D4T<R> b) { return -(b - a); }
template <class R> __device__ __forceinline__ D4T<R> operator/(D4T<R> a, D4T<R> b) {
  const R q = a.v / b.v;
  const R ib = R(1) / b.v;
  return D4T<R>{q, {(a.d[0] - q * b.d[0]) * ib, (a.d[1] - q * b.d[1]) * ib, (a.d[2] - q * b.d[2]) * ib,
                    (a.d[3] - q * b.d[3]) * ib}};
}
template <class R> __device__ __forceinline__ D4T<R> operator/(R a, D4T<R> b) { return d4c(a) / b; }
template <class R> __device__ __forceinline__ D4T<R> dsqrt(D4T<R> a) {
  const R r = sqrt(a.v);
  const R k = r > R(0) ? R(0.5) / r : R(0);
  return D4T<R>{r, {a.d[0] * k, a.d[1] * k, a.d[2] * k, a.d[3] * k}};
}
__device__ __forceinline__ float val(float a) { return a; }
__device__ __forceinline__ double val(double a) { return a; }
template <class R> __device__ __forceinline__ R val(D4T<R> a) { return a.v; }
__device__ __forceinline__ float dsqrt(float a) { return sqrtf(a); }
__device__ __forceinline__ double dsqrt(double a) { return sqrt(a); }

// the real type of T (T itself, or a dual's value type)
template <class T> struct RealOf { using type = T; };
template <class R> struct RealOf<D4T<R>> { using type = R; };

// scalar constant in the type T
template <class T> __device__ __forceinline__ T tconst(typename RealOf<T>::type v) { return v; }
template <> __device__ __forceinline__ D4T<float> tconst<D4T<float>>(float v) { return d4c(v); }
template <> __device__ __forceinline__ D4T<double> tconst<D4T<double>>(double v) { return d4c(v); }

template <class T, class R>
__device__ __forceinline__ T tmax(T a, R b) { return val(a) > b ? a : tconst<T>(b); }
template <class T, class R>
__device__ __forceinline__ T tmin(T a, R b) { return val(a) < b ? a : tconst<T>(b); }

// Phi of the P2G material update (mpm_sim.py:206-233), for the adjoint.
// A = F* = (I + dt C) F row-major.  Outputs F_out (the stored deformation
// gradient), the Kirchhoff stress tau (without the dt * p_vol scaling) and
// J; the muscle's active term enters as pressure * J * d d^T.
template <class T>
__device__ __forceinline__ void jf_phi(const T A[4], int mt, typename RealOf<T>::type mu,
                                       typename RealOf<T>::type la, typename RealOf<T>::type pressure,
                                       float2 fiber, T Fout[4], T tau[4], T& J) {
  using R = typename RealOf<T>::type;
  const R fdx = fiber.x, fdy = fiber.y;
  const T x = A[0] + A[3];
  const T y = A[2] - A[1];
  const T scale = tconst<T>(R(1)) / dsqrt(x * x + y * y);
  const T c = x * scale, s = y * scale, ms = -s;
  const T S00 = c * A[0] + s * A[2];
  const T S01 = c * A[1] + s * A[3];
  const T S11 = ms * A[1] + c * A[3];
  T cc, ss, s1, s2;
  const R s01v = val(S01);
  if ((s01v < R(0) ? -s01v : s01v) < R(1e-5)) {
    cc = tconst<T>(R(1));
    ss = tconst<T>(R(0));
    s1 = S00;
    s2 = S11;
  } else {
    const T tao = R(0.5) * (S00 - S11);
    const T w = dsqrt(tao * tao + S01 * S01);
    const T t = val(tao) > R(0) ? S01 / (tao + w) : S01 / (tao - w);
    cc = tconst<T>(R(1)) / dsqrt(t * t + R(1));
    ss = -t * cc;
    s1 = (cc * cc * S00 - R(2) * cc * ss * S01) + ss * ss * S11;
    s2 = (ss * ss * S00 + R(2) * cc * ss * S01) + cc * cc * S11;
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
  s1 = tmax(s1, R(1e-6));
  s2 = tmax(s2, R(1e-6));
  if (mt == 2) {
    s1 = tmin(tmax(s1, R(1 - 5e-3)), R(1 + 5e-3));
    s2 = tmin(tmax(s2, R(1 - 5e-3)), R(1 + 5e-3));
  }
  J = s1 * s2;
  if (mt == 0) {
    const T sj = dsqrt(J);
    Fout[0] = sj; Fout[1] = tconst<T>(R(0)); Fout[2] = tconst<T>(R(0)); Fout[3] = sj;
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
  const R twomu = R(2) * mu;
  const T E00 = twomu * (Fout[0] - R00), E01 = twomu * (Fout[1] - R01);
  const T E10 = twomu * (Fout[2] - R10), E11 = twomu * (Fout[3] - R11);
  const T diag = la * J * (J - R(1));
  tau[0] = (E00 * Fout[0] + E01 * Fout[1]) + diag;
  tau[1] = E00 * Fout[2] + E01 * Fout[3];
  tau[2] = E10 * Fout[0] + E11 * Fout[1];
  tau[3] = (E10 * Fout[2] + E11 * Fout[3]) + diag;
  if (mt == 3) {
    tau[0] = tau[0] + (fdx * fdx * pressure) * J;
    tau[1] = tau[1] + (fdx * fdy * pressure) * J;
    tau[2] = tau[2] + (fdy * fdx * pressure) * J;
    tau[3] = tau[3] + (fdy * fdy * pressure) * J;
  }
}
