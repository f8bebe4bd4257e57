// cc_device.cuh -- device building blocks shared by the sm_100a kernels.
//
// Everything here is compiled with --fmad=false and IEEE division / square root, so each
// expression rounds exactly as the reference's Julia code does on the CPU (Julia contracts no
// a*b+c unless asked). Expression order follows the reference line by line (StaticArrays left
// folds, elementwise division); the citations are to the reference files.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include "../../include/cutcell_b200.h"

namespace ccd {

template <class T> struct Eps;
template <> struct Eps<float> { static __device__ __forceinline__ float v() { return 1.1920928955078125e-07f; } };
template <> struct Eps<double> { static __device__ __forceinline__ double v() { return 2.220446049250313e-16; } };

template <class T> __device__ __forceinline__ T qnan();
template <> __device__ __forceinline__ float qnan<float>() { return __int_as_float(0x7fc00000); }
template <> __device__ __forceinline__ double qnan<double>() { return __longlong_as_double(0x7ff8000000000000ll); }

// ---------------------------------------------------------------------------------------------
// Op-tape (include/cutcell_b200.h). The tape is copied into shared memory once per CTA; every
// lane reads the same op at the same time, so the reads are broadcasts.
template <class T>
struct STape {
  const cc_op* ops;
  const T* p;
  int n_ops;
};

// Forward-mode dual: the value and its gradient in D coordinates (the PLIC normal).
template <class T, int D>
struct Dual {
  T v;
  T g[D];
};
template <class T> __device__ __forceinline__ T val(T x) { return x; }
template <class T, int D> __device__ __forceinline__ T val(const Dual<T, D>& x) { return x.v; }

template <class S, class T> struct Lift { static __device__ __forceinline__ S c(T x) { return x; } };
template <class T, int D> struct Lift<Dual<T, D>, T> {
  static __device__ __forceinline__ Dual<T, D> c(T x) {
    Dual<T, D> r; r.v = x;
#pragma unroll
    for (int i = 0; i < D; ++i) r.g[i] = T(0);
    return r;
  }
};

template <class T, int D>
__device__ __forceinline__ Dual<T, D> operator+(const Dual<T, D>& a, const Dual<T, D>& b) {
  Dual<T, D> r; r.v = a.v + b.v;
#pragma unroll
  for (int i = 0; i < D; ++i) r.g[i] = a.g[i] + b.g[i];
  return r; }
template <class T, int D>
__device__ __forceinline__ Dual<T, D> operator-(const Dual<T, D>& a, const Dual<T, D>& b) {
  Dual<T, D> r; r.v = a.v - b.v;
#pragma unroll
  for (int i = 0; i < D; ++i) r.g[i] = a.g[i] - b.g[i];
  return r; }
template <class T, int D>
__device__ __forceinline__ Dual<T, D> operator-(const Dual<T, D>& a) {
  Dual<T, D> r; r.v = -a.v;
#pragma unroll
  for (int i = 0; i < D; ++i) r.g[i] = -a.g[i];
  return r; }
template <class T, int D>
__device__ __forceinline__ Dual<T, D> operator*(const Dual<T, D>& a, const Dual<T, D>& b) {
  Dual<T, D> r; r.v = a.v * b.v;
#pragma unroll
  for (int i = 0; i < D; ++i) r.g[i] = a.g[i] * b.v + a.v * b.g[i];
  return r; }
template <class T, int D>
__device__ __forceinline__ Dual<T, D> operator/(const Dual<T, D>& a, const Dual<T, D>& b) {
  Dual<T, D> r; r.v = a.v / b.v;
  const T bb = b.v * b.v;
#pragma unroll
  for (int i = 0; i < D; ++i) r.g[i] = (a.g[i] * b.v - a.v * b.g[i]) / bb;
  return r; }
template <class T, int D>
__device__ __forceinline__ Dual<T, D> operator+(const Dual<T, D>& a, T c) { Dual<T, D> r = a; r.v = a.v + c; return r; }
template <class T, int D>
__device__ __forceinline__ Dual<T, D> operator-(const Dual<T, D>& a, T c) { Dual<T, D> r = a; r.v = a.v - c; return r; }
template <class T, int D>
__device__ __forceinline__ Dual<T, D> operator-(T c, const Dual<T, D>& a) { Dual<T, D> r = -a; r.v = c - a.v; return r; }
template <class T, int D>
__device__ __forceinline__ Dual<T, D> operator*(T c, const Dual<T, D>& a) {
  Dual<T, D> r; r.v = c * a.v;
#pragma unroll
  for (int i = 0; i < D; ++i) r.g[i] = c * a.g[i];
  return r; }
template <class T, int D>
__device__ __forceinline__ Dual<T, D> operator*(const Dual<T, D>& a, T c) {
  Dual<T, D> r; r.v = a.v * c;
#pragma unroll
  for (int i = 0; i < D; ++i) r.g[i] = a.g[i] * c;
  return r; }
template <class T, int D>
__device__ __forceinline__ Dual<T, D> operator/(const Dual<T, D>& a, T c) {
  Dual<T, D> r; r.v = a.v / c;
#pragma unroll
  for (int i = 0; i < D; ++i) r.g[i] = a.g[i] / c;
  return r; }
template <class T, int D>
__device__ __forceinline__ Dual<T, D> dsqrt(const Dual<T, D>& a) {
  Dual<T, D> r; r.v = sqrt(a.v);
  const T two_s = T(2) * r.v;
#pragma unroll
  for (int i = 0; i < D; ++i) r.g[i] = a.g[i] / two_s;
  return r; }
template <class T, int D>
__device__ __forceinline__ Dual<T, D> dabs(const Dual<T, D>& a) {
  const T sg = a.v > T(0) ? T(1) : (a.v < T(0) ? T(-1) : T(0));
  Dual<T, D> r; r.v = fabs(a.v);
#pragma unroll
  for (int i = 0; i < D; ++i) r.g[i] = sg * a.g[i];
  return r; }
template <class T, int D>
__device__ __forceinline__ Dual<T, D> dsin(const Dual<T, D>& a) {
  Dual<T, D> r; r.v = sin(a.v); const T c = cos(a.v);
#pragma unroll
  for (int i = 0; i < D; ++i) r.g[i] = c * a.g[i];
  return r; }
template <class T, int D>
__device__ __forceinline__ Dual<T, D> dcos(const Dual<T, D>& a) {
  Dual<T, D> r; r.v = cos(a.v); const T s = -sin(a.v);
#pragma unroll
  for (int i = 0; i < D; ++i) r.g[i] = s * a.g[i];
  return r; }
template <class T, int D>
__device__ __forceinline__ Dual<T, D> datan2(const Dual<T, D>& y, const Dual<T, D>& x) {
  Dual<T, D> r; r.v = atan2(y.v, x.v);
  const T den = x.v * x.v + y.v * y.v;
#pragma unroll
  for (int i = 0; i < D; ++i) r.g[i] = (x.v * y.g[i] - y.v * x.g[i]) / den;
  return r; }

__device__ __forceinline__ float dsqrt(float a) { return sqrtf(a); }
__device__ __forceinline__ double dsqrt(double a) { return sqrt(a); }
__device__ __forceinline__ float dabs(float a) { return fabsf(a); }
__device__ __forceinline__ double dabs(double a) { return fabs(a); }
__device__ __forceinline__ float dsin(float a) { return sinf(a); }
__device__ __forceinline__ double dsin(double a) { return sin(a); }
__device__ __forceinline__ float dcos(float a) { return cosf(a); }
__device__ __forceinline__ double dcos(double a) { return cos(a); }
__device__ __forceinline__ float datan2(float y, float x) { return atan2f(y, x); }
__device__ __forceinline__ double datan2(double y, double x) { return atan2(y, x); }

// Primitive parameter blocks start on a 4-element boundary of the tape's parameter array (the
// host packs them so), so a block is read with 16-byte vector loads.
__device__ __forceinline__ void ldq(const float* p, float* o) {
  const float4 t = *reinterpret_cast<const float4*>(p);
  o[0] = t.x; o[1] = t.y; o[2] = t.z; o[3] = t.w;
}
__device__ __forceinline__ void ldq(const double* p, double* o) {
  const double2 a = *reinterpret_cast<const double2*>(p);
  const double2 b = *reinterpret_cast<const double2*>(p + 2);
  o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y;
}

// One primitive at the point x (SDFLibrary's sdf_value / get_sdf stand-ins).
template <class T, int D, class S>
__device__ __forceinline__ S tape_prim(const cc_op op, const T* __restrict__ p, const S* x) {
  const T* b = p + op.poff;
  switch (op.opcode) {
    case CC_OP_SPHERE: {
      T c[4];
      ldq(b, c);
      S u = (x[0] - c[0]) * (x[0] - c[0]);
#pragma unroll
      for (int a = 1; a < D; ++a) u = u + (x[a] - c[a]) * (x[a] - c[a]);
      return dsqrt(u) - c[D];
    }
    case CC_OP_BOX: {
      T c[8];
      ldq(b, c);
      if (D == 3) ldq(b + 4, c + 4);
      S q[D];
#pragma unroll
      for (int a = 0; a < D; ++a) q[a] = dabs(x[a] - c[a]) - c[D + a];
      const S zero = Lift<S, T>::c(T(0));
      S qa = val(q[0]) > T(0) ? q[0] : zero;
      S u = qa * qa;
#pragma unroll
      for (int a = 1; a < D; ++a) { qa = val(q[a]) > T(0) ? q[a] : zero; u = u + qa * qa; }
      const S outside = dsqrt(u);
      S m = q[0];
#pragma unroll
      for (int a = 1; a < D; ++a) m = val(q[a]) > val(m) ? q[a] : m;
      const S inside = val(m) < T(0) ? m : zero;
      return outside + inside;
    }
    case CC_OP_TORUS:
      if constexpr (D == 3) {
        T c[16];
        ldq(b, c); ldq(b + 4, c + 4); ldq(b + 8, c + 8); ldq(b + 12, c + 12);
        const T* R = c + 3;
        const S d0 = x[0] - c[0], d1 = x[1] - c[1], d2 = x[2] - c[2];
        const S l0 = R[0] * d0 + R[1] * d1 + R[2] * d2;
        const S l1 = R[3] * d0 + R[4] * d1 + R[5] * d2;
        const S l2 = R[6] * d0 + R[7] * d1 + R[8] * d2;
        const S qx = dsqrt(l0 * l0 + l1 * l1) - c[12];
        return dsqrt(qx * qx + l2 * l2) - c[13];
      } else {
        return Lift<S, T>::c(qnan<T>());
      }
    case CC_OP_PLANE: {
      T c[8];
      ldq(b, c);
      if (D == 3) ldq(b + 4, c + 4);
      S s = c[D] * (x[0] - c[0]);
#pragma unroll
      for (int a = 1; a < D; ++a) s = s + c[D + a] * (x[a] - c[a]);
      return s;
    }
    case CC_OP_TRIG: {
      T q[8];
      ldq(b, q);
      if (D == 3) ldq(b + 4, q + 4);
      S s = q[0] * dsin(q[1] * x[0]);
#pragma unroll
      for (int a = 1; a < D; ++a) s = s * dsin(q[1 + a] * x[a]);
      return s + q[1 + D];
    }
    case CC_OP_CONST:
      return Lift<S, T>::c(b[0]);
    case CC_OP_STAR:
      if constexpr (D == 2) {
        T q[16];
        ldq(b, q); ldq(b + 4, q + 4); ldq(b + 8, q + 8); ldq(b + 12, q + 12);
        const S dx = x[0] - q[0], dy = x[1] - q[1];
        const S rad = dsqrt(dx * dx + dy * dy);
        const S th = datan2(dy, dx);
        S r = Lift<S, T>::c(q[2]);
        for (int k = 2; k <= 6; ++k) r = r + q[3 + (k - 2)] * dcos(T(k) * th + q[8 + (k - 2)]);
        return rad - r;
      } else {
        return Lift<S, T>::c(qnan<T>());
      }
    default:
      return Lift<S, T>::c(qnan<T>());
  }
}

template <class T, class S>
__device__ __forceinline__ S tape_combine(int mode, const S& top, const S& v, T k) {
  switch (mode) {
    case CC_COMB_MIN: return val(v) < val(top) ? v : top;
    case CC_COMB_MAX: return val(v) > val(top) ? v : top;
    case CC_COMB_SUB: { const S w = -v; return val(w) > val(top) ? w : top; }
    case CC_COMB_SMIN: {
      const S ad = dabs(top - v);
      const S hk = k - ad;
      const S zero = Lift<S, T>::c(T(0));
      const S h = (val(hk) > T(0) ? hk : zero) / k;
      const S m = val(v) < val(top) ? v : top;
      return m - ((h * h) * k) * T(0.25);
    }
    default: return v;
  }
}

// Postfix evaluation. The top of the stack lives in a register; only nested CSG (a combinator
// whose operand is itself a combinator) touches the local-memory stack below it.
template <class T, int D, class S>
__device__ __forceinline__ S tape_eval(const STape<T>& t, const S* x) {
  S acc = Lift<S, T>::c(T(0));
  S st[CC_TAPE_MAX_STACK];
  int sp = 0;  // entries below acc
  bool have = false;
  for (int i = 0; i < t.n_ops; ++i) {
    const cc_op op = t.ops[i];
    S v;
    if (op.opcode == CC_OP_NONE) {
      if (op.combine == CC_COMB_NEG) { acc = -acc; continue; }
      v = acc;
      acc = st[--sp];
    } else {
      v = tape_prim<T, D, S>(op, t.p, x);
    }
    if (op.combine == CC_COMB_PUSH) {
      if (have) st[sp++] = acc;
      acc = v;
      have = true;
    } else {
      acc = tape_combine<T, S>(op.combine, acc, v, op.combine == CC_COMB_SMIN ? t.p[op.kparam] : T(0));
    }
  }
  return acc;
}

// Op-major evaluation of one tape at NB points at once (scalar T only): each op's dispatch and
// parameter loads are paid once for all NB points, and the NB dependency chains interleave.
// Per point the arithmetic is exactly tape_eval's, in the same order.
template <class T, int D, int NB>
__device__ __forceinline__ void tape_prim_multi(const cc_op op, const T* __restrict__ p, const T (&x)[NB][D], T (&v)[NB]) {
  const T* b = p + op.poff;
  switch (op.opcode) {
    case CC_OP_SPHERE: {
      T c[4];
      ldq(b, c);
#pragma unroll
      for (int q = 0; q < NB; ++q) {
        T u = (x[q][0] - c[0]) * (x[q][0] - c[0]);
#pragma unroll
        for (int a = 1; a < D; ++a) u = u + (x[q][a] - c[a]) * (x[q][a] - c[a]);
        v[q] = dsqrt(u) - c[D];
      }
      return;
    }
    case CC_OP_BOX: {
      T c[8];
      ldq(b, c);
      if (D == 3) ldq(b + 4, c + 4);
#pragma unroll
      for (int q = 0; q < NB; ++q) {
        T qq[D];
#pragma unroll
        for (int a = 0; a < D; ++a) qq[a] = dabs(x[q][a] - c[a]) - c[D + a];
        T qa = qq[0] > T(0) ? qq[0] : T(0);
        T u = qa * qa;
#pragma unroll
        for (int a = 1; a < D; ++a) { qa = qq[a] > T(0) ? qq[a] : T(0); u = u + qa * qa; }
        const T outside = dsqrt(u);
        T m = qq[0];
#pragma unroll
        for (int a = 1; a < D; ++a) m = qq[a] > m ? qq[a] : m;
        const T inside = m < T(0) ? m : T(0);
        v[q] = outside + inside;
      }
      return;
    }
    case CC_OP_TORUS:
      if constexpr (D == 3) {
        T c[16];
        ldq(b, c); ldq(b + 4, c + 4); ldq(b + 8, c + 8); ldq(b + 12, c + 12);
        const T* R = c + 3;
#pragma unroll
        for (int q = 0; q < NB; ++q) {
          const T d0 = x[q][0] - c[0], d1 = x[q][1] - c[1], d2 = x[q][2] - c[2];
          const T l0 = R[0] * d0 + R[1] * d1 + R[2] * d2;
          const T l1 = R[3] * d0 + R[4] * d1 + R[5] * d2;
          const T l2 = R[6] * d0 + R[7] * d1 + R[8] * d2;
          const T qx = dsqrt(l0 * l0 + l1 * l1) - c[12];
          v[q] = dsqrt(qx * qx + l2 * l2) - c[13];
        }
        return;
      }
      break;
    case CC_OP_PLANE: {
      T c[8];
      ldq(b, c);
      if (D == 3) ldq(b + 4, c + 4);
#pragma unroll
      for (int q = 0; q < NB; ++q) {
        T s = c[D] * (x[q][0] - c[0]);
#pragma unroll
        for (int a = 1; a < D; ++a) s = s + c[D + a] * (x[q][a] - c[a]);
        v[q] = s;
      }
      return;
    }
    case CC_OP_TRIG: {
      T c[8];
      ldq(b, c);
      if (D == 3) ldq(b + 4, c + 4);
#pragma unroll
      for (int q = 0; q < NB; ++q) {
        T s = c[0] * dsin(c[1] * x[q][0]);
#pragma unroll
        for (int a = 1; a < D; ++a) s = s * dsin(c[1 + a] * x[q][a]);
        v[q] = s + c[1 + D];
      }
      return;
    }
    case CC_OP_CONST: {
      const T c = b[0];
#pragma unroll
      for (int q = 0; q < NB; ++q) v[q] = c;
      return;
    }
    default:
      break;
  }
  // primitives without a multi-point form (and invalid opcodes) fall back point by point
#pragma unroll
  for (int q = 0; q < NB; ++q) v[q] = tape_prim<T, D, T>(op, p, x[q]);
}

template <class T, int D, int NB>
__device__ __forceinline__ void tape_eval_multi(const STape<T>& t, const T (&x)[NB][D], T (&out)[NB]) {
  T acc[NB];
#pragma unroll
  for (int q = 0; q < NB; ++q) acc[q] = T(0);
  T st[CC_TAPE_MAX_STACK][NB];
  int sp = 0;
  bool have = false;
  for (int i = 0; i < t.n_ops; ++i) {
    const cc_op op = t.ops[i];
    T v[NB];
    if (op.opcode == CC_OP_NONE) {
      if (op.combine == CC_COMB_NEG) {
#pragma unroll
        for (int q = 0; q < NB; ++q) acc[q] = -acc[q];
        continue;
      }
      --sp;
#pragma unroll
      for (int q = 0; q < NB; ++q) { v[q] = acc[q]; acc[q] = st[sp][q]; }
    } else {
      tape_prim_multi<T, D, NB>(op, t.p, x, v);
    }
    switch (op.combine) {
      case CC_COMB_PUSH:
        if (have) {
#pragma unroll
          for (int q = 0; q < NB; ++q) st[sp][q] = acc[q];
          ++sp;
        }
#pragma unroll
        for (int q = 0; q < NB; ++q) acc[q] = v[q];
        have = true;
        break;
      case CC_COMB_MIN:
#pragma unroll
        for (int q = 0; q < NB; ++q) acc[q] = v[q] < acc[q] ? v[q] : acc[q];
        break;
      case CC_COMB_MAX:
#pragma unroll
        for (int q = 0; q < NB; ++q) acc[q] = v[q] > acc[q] ? v[q] : acc[q];
        break;
      default: {
        const T k = op.combine == CC_COMB_SMIN ? t.p[op.kparam] : T(0);
#pragma unroll
        for (int q = 0; q < NB; ++q) acc[q] = tape_combine<T, T>(op.combine, acc[q], v[q], k);
      }
    }
  }
#pragma unroll
  for (int q = 0; q < NB; ++q) out[q] = acc[q];
}

// Copy a packed tape (ops, padded to 16 bytes, then the parameter blocks narrowed to T, each
// starting on a 4-element boundary) from global into shared memory.
__host__ __device__ __forceinline__ int tape_ops_bytes(int n_ops) { return ((n_ops * int(sizeof(cc_op)) + 15) / 16) * 16; }
template <class T>
__device__ __forceinline__ STape<T> load_tape(const unsigned char* __restrict__ gtape, int n_ops, int n_params,
                                              unsigned char* smem) {
  const int bytes = tape_ops_bytes(n_ops) + n_params * int(sizeof(T));
  const int words = (bytes + 7) / 8;
  const unsigned long long* src = reinterpret_cast<const unsigned long long*>(gtape);
  unsigned long long* dst = reinterpret_cast<unsigned long long*>(smem);
  for (int w = threadIdx.x; w < words; w += blockDim.x) dst[w] = __ldg(src + w);
  STape<T> t;
  t.ops = reinterpret_cast<const cc_op*>(smem);
  t.p = reinterpret_cast<const T*>(smem + tape_ops_bytes(n_ops));
  t.n_ops = n_ops;
  return t;
}

// ---------------------------------------------------------------------------------------------
// Pruning a union of spheres to a region. For a tape that is a union (mode 1: PUSH then MIN) or
// smooth union (mode 2: PUSH then SMIN) of spheres, and a box containing every point a CTA will
// evaluate, the ops that cannot change any of those values are dropped:
//  * union: sphere i is dropped when its smallest value over the box exceeds the largest value of
//    some other sphere there -- it is then strictly above the minimum everywhere, never selected,
//    and the minimum (value and gradient) is bit-identical without it;
//  * smooth union: sphere i (i > 0) is dropped when its smallest value exceeds, by its smoothing k,
//    the largest value over the box of every earlier sphere's minimum -- then the smooth-min step
//    sees |top - v| >= k, h = 0, and returns the running value unchanged, bit for bit.
// The bounds carry a margin of 16 eps(T) times the magnitudes involved, so T's rounding of the
// evaluation can not cross them. All threads call this; it returns the kept op count and writes
// the kept ops (the first one's combine made PUSH) to `out`. `ls`, `us`: n_ops doubles each.
template <class T, int D>
__device__ int prune_union(const STape<T>& t, int mode, const double lo[D], const double hi[D], double* ls, double* us,
                           cc_op* out, int* count) {
  const int n = t.n_ops;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const T* p = t.p + t.ops[i].poff;
    double dmin2 = 0.0, dmax2 = 0.0, mag = fabs(double(p[D])) + 1.0;
#pragma unroll
    for (int a = 0; a < D; ++a) {
      const double c = p[a];
      const double below = lo[a] - c, above = c - hi[a];
      const double dn = below > 0.0 ? below : (above > 0.0 ? above : 0.0);
      const double dx = fabs(lo[a] - c) > fabs(hi[a] - c) ? fabs(lo[a] - c) : fabs(hi[a] - c);
      dmin2 += dn * dn;
      dmax2 += dx * dx;
      mag += fabs(c) + (fabs(lo[a]) > fabs(hi[a]) ? fabs(lo[a]) : fabs(hi[a]));
    }
    const double r = p[D];
    const double margin = 16.0 * double(Eps<T>::v()) * (mag + sqrt(dmax2));
    ls[i] = sqrt(dmin2) - r - margin;
    us[i] = sqrt(dmax2) - r + margin;
  }
  __syncthreads();
  if (n <= int(blockDim.x) && blockDim.x <= 1024) {
    // one op per thread: block reductions and scans, then an order-preserving compaction
    __shared__ double s_val[32];
    __shared__ int s_idx[32];
    __shared__ int s_cnt[32];
    const int i = threadIdx.x, lane = i & 31, w = i >> 5, nw = (blockDim.x + 31) >> 5;
    const double u = i < n ? us[i] : 1.0e300;
    bool keep = false;
    if (mode == 1) {
      // the smallest upper bound, its op, and the smallest of the others
      double v = u;
      int vi = i;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, v, o);
        const int oi = __shfl_xor_sync(0xffffffffu, vi, o);
        if (ov < v || (ov == v && oi < vi)) { v = ov; vi = oi; }
      }
      if (lane == 0) { s_val[w] = v; s_idx[w] = vi; }
      __syncthreads();
      double mn = s_val[0];
      int jm = s_idx[0];
      for (int q = 1; q < nw; ++q)
        if (s_val[q] < mn || (s_val[q] == mn && s_idx[q] < jm)) { mn = s_val[q]; jm = s_idx[q]; }
      __syncthreads();
      double v2 = i == jm ? 1.0e300 : u;
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, v2, o);
        v2 = ov < v2 ? ov : v2;
      }
      if (lane == 0) s_val[w] = v2;
      __syncthreads();
      double mn2 = s_val[0];
      for (int q = 1; q < nw; ++q) mn2 = s_val[q] < mn2 ? s_val[q] : mn2;
      keep = i < n && !(ls[i] > (i == jm ? mn2 : mn));
    } else {
      // the exclusive prefix minimum of the upper bounds
      double v = u;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const double ov = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v = ov < v ? ov : v;
      }
      if (lane == 31) s_val[w] = v;
      __syncthreads();
      double before = 1.0e300;  // the minimum over the earlier warps
      for (int q = 0; q < w; ++q) before = s_val[q] < before ? s_val[q] : before;
      double up = __shfl_up_sync(0xffffffffu, v, 1);
      if (lane == 0) up = 1.0e300;
      const double prefix = up < before ? up : before;  // min over ops 0..i-1
      if (i < n) {
        if (i == 0) keep = true;
        else {
          const double k = t.p[t.ops[i].kparam];
          const double kmargin = 16.0 * double(Eps<T>::v()) * (fabs(k) + fabs(prefix) + fabs(ls[i]) + 1.0);
          keep = !(ls[i] >= prefix + k + kmargin);
        }
      }
      __syncthreads();
    }
    const unsigned b = __ballot_sync(0xffffffffu, keep);
    if (lane == 0) s_cnt[w] = __popc(b);
    __syncthreads();
    int pos = __popc(b & ((1u << lane) - 1u));
    int total = 0;
    for (int q = 0; q < nw; ++q) {
      if (q < w) pos += s_cnt[q];
      total += s_cnt[q];
    }
    if (keep) {
      cc_op op = t.ops[i];
      if (pos == 0) op.combine = CC_COMB_PUSH;
      out[pos] = op;
    }
    if (i == 0) *count = total;
    __syncthreads();
    return *count;
  }
  if (threadIdx.x == 0) {
    int m = 0;
    if (mode == 1) {
      int jm = 0;
      for (int j = 1; j < n; ++j) if (us[j] < us[jm]) jm = j;
      double u2 = 1.0e300;
      for (int j = 0; j < n; ++j) if (j != jm && us[j] < u2) u2 = us[j];
      for (int i = 0; i < n; ++i) {
        if (ls[i] > (i == jm ? u2 : us[jm])) continue;
        cc_op op = t.ops[i];
        if (m == 0) op.combine = CC_COMB_PUSH;
        out[m++] = op;
      }
    } else {
      double prefix = us[0];
      out[m++] = t.ops[0];
      for (int i = 1; i < n; ++i) {
        const double k = t.p[t.ops[i].kparam];
        const double kmargin = 16.0 * double(Eps<T>::v()) * (fabs(k) + fabs(prefix) + fabs(ls[i]) + 1.0);
        if (!(ls[i] >= prefix + k + kmargin)) out[m++] = t.ops[i];
        if (us[i] < prefix) prefix = us[i];
      }
    }
    *count = m;
  }
  __syncthreads();
  return *count;
}

// Shared-memory places of prune_union's output and scratch, after a tape loaded at `base`.
struct PruneSmem {
  int ops, ls, us, end;
  template <class DT>
  __host__ __device__ static PruneSmem of(const DT& tape, int base) {
    PruneSmem p;
    p.ops = base + ((tape.bytes_len + 15) / 16) * 16;
    p.ls = p.ops + ((tape.n_ops * int(sizeof(cc_op)) + 15) / 16) * 16;
    p.us = p.ls + tape.n_ops * 8;
    p.end = p.us + tape.n_ops * 8;
    return p;
  }
};

// ---------------------------------------------------------------------------------------------
// CartesianMeshes stand-ins: node and centroid coordinates, the plane-cube clip.
template <class T> __device__ __forceinline__ T node_coord(T x0, T d, long long i) { return x0 + T(i) * d; }
template <class T> __device__ __forceinline__ T centroid_coord(T x0, T d, long long i) {
  return x0 + T(double(i) + 0.5) * d;
}

// Mixed precision (CC_MIXED): Float32 storage and bulk arithmetic with FP64 islands. The
// template flag MX selects them; it is only ever set with T = float.
//  * the edge root phi_a / (phi_a - phi_b) in FP64 when the FP32 denominator is below 2^-100,
//    where FP32 quotients of (near-)subnormal values lose bits;
//  * the asymptotic deciders (test_face / test_interior): products of FP32 values are exact in
//    FP64, so a decider's sign is the exact sign of its FP32 inputs' determinant;
//  * the plane-cube clip of PLIC (gvf2 / gvf3) evaluated in FP64 and rounded once.
constexpr float MIXED_TINY = 7.8886090522101181e-31f;  // 2^-100

// _open_fraction, src/marching_squares/marching_squares.jl:192-198
template <class T, bool MX = false>
__device__ __forceinline__ T open_fraction(T pa, T pb) {
  const bool fa = pa >= T(0), fb = pb >= T(0);
  if (fa && fb) return T(1);
  if (!fa && !fb) return T(0);
  if constexpr (MX) {
    const T den = fa ? pa - pb : pb - pa;
    if (fabs(den) < T(MIXED_TINY))
      return T(fa ? double(pa) / (double(pa) - double(pb)) : double(pb) / (double(pb) - double(pa)));
  }
  return fa ? pa / (pa - pb) : pb / (pb - pa);
}

// Solid fraction of the unit square {n . xi <= a} (Scardovelli & Zaleski 2000).
template <class T>
__device__ __forceinline__ T gvf2(T n1, T n2, T a) {
  T m1 = fabs(n1), m2 = fabs(n2);
  T alpha = a;
  if (n1 < T(0)) alpha = alpha + m1;
  if (n2 < T(0)) alpha = alpha + m2;
  const T s = m1 + m2;
  if (!(s > T(0))) return alpha >= T(0) ? T(1) : T(0);
  // a plane that misses the square: alpha / s <= 0 exactly when alpha <= 0, and alpha / s >= 1 when
  // alpha >= s (rounding is monotone), so these are the returns below without the divisions
  if (alpha <= T(0)) return T(0);
  if (alpha >= s) return T(1);
  m1 = m1 / s; m2 = m2 / s; alpha = alpha / s;
  if (alpha <= T(0)) return T(0);
  if (alpha >= T(1)) return T(1);
  const bool flip = alpha > T(0.5);
  if (flip) alpha = T(1) - alpha;
  if (m1 > m2) { const T t = m1; m1 = m2; m2 = t; }
  T v;
  if (alpha < m1) v = (alpha * alpha) / (T(2) * m1 * m2);
  else v = (alpha - T(0.5) * m1) / m2;
  return flip ? T(1) - v : v;
}

// Solid fraction of the unit cube {n . xi <= a} (Scardovelli & Zaleski 2000, with the
// alpha^3 - (alpha - m1)^3 difference expanded so no branch divides a cancellation by a small m1).
template <class T>
__device__ __forceinline__ T gvf3(T n1, T n2, T n3, T a) {
  T m0 = fabs(n1), m1_ = fabs(n2), m2_ = fabs(n3);
  T alpha = a;
  if (n1 < T(0)) alpha = alpha + m0;
  if (n2 < T(0)) alpha = alpha + m1_;
  if (n3 < T(0)) alpha = alpha + m2_;
  const T s = (m0 + m1_) + m2_;
  if (!(s > T(0))) return alpha >= T(0) ? T(1) : T(0);
  // a plane that misses the cube: the returns below without the divisions (as in gvf2)
  if (alpha <= T(0)) return T(0);
  if (alpha >= s) return T(1);
  m0 = m0 / s; m1_ = m1_ / s; m2_ = m2_ / s; alpha = alpha / s;
  if (alpha <= T(0)) return T(0);
  if (alpha >= T(1)) return T(1);
  const bool flip = alpha > T(0.5);
  if (flip) alpha = T(1) - alpha;
  T t;
  if (m0 > m1_) { t = m0; m0 = m1_; m1_ = t; }
  if (m1_ > m2_) { t = m1_; m1_ = m2_; m2_ = t; }
  if (m0 > m1_) { t = m0; m0 = m1_; m1_ = t; }
  const T m1 = m0, m2 = m1_, m3 = m2_;
  const T m12 = m1 + m2;
  T v;
  if (alpha < m1) {
    v = (alpha * alpha * alpha) / (T(6) * m1 * m2 * m3);
  } else {
    const T core = (T(3) * alpha * alpha - T(3) * alpha * m1 + m1 * m1) / (T(6) * m2 * m3);
    if (alpha < m2) {
      v = core;
    } else if (alpha < (m12 < m3 ? m12 : m3)) {
      const T u = alpha - m2;
      v = core - (u * u * u) / (T(6) * m1 * m2 * m3);
    } else if (m3 < m12) {
      const T u = alpha - m2, w = alpha - m3;
      v = core - (u * u * u + w * w * w) / (T(6) * m1 * m2 * m3);
    } else {
      v = (T(2) * alpha - m12) / (T(2) * m3);
    }
  }
  return flip ? T(1) - v : v;
}

// The plane-cube clips under a precision policy: with MX (T = float), evaluated in FP64 from the
// FP32 arguments and rounded once.
template <class T, bool MX>
__device__ __forceinline__ T gvf2m(T n1, T n2, T a) {
  if constexpr (MX) return T(gvf2<double>(double(n1), double(n2), double(a)));
  else return gvf2<T>(n1, n2, a);
}
template <class T, bool MX>
__device__ __forceinline__ T gvf3m(T n1, T n2, T n3, T a) {
  if constexpr (MX) return T(gvf3<double>(double(n1), double(n2), double(n3), double(a)));
  else return gvf3<T>(n1, n2, n3, a);
}

}  // namespace ccd
