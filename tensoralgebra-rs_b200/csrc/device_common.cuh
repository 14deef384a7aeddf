// Small device helpers shared by the kernels: element traits and the
// alpha/beta/conjugation epilogue of one output element.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "kernels.cuh"

namespace tprims {
namespace dev {

template <class R>
struct Cplx {
  R re, im;
};

// Storage element of a dtype: real R or interleaved complex of R.
template <class R, bool CPLX>
struct Elem;
template <class R>
struct Elem<R, false> {
  using type = R;
  __device__ static inline void load(const type* p, R& re, R& im) {
    re = *p;
    im = R(0);
  }
  __device__ static inline void store(type* p, R re, R) { *p = re; }
};
template <class R>
struct Elem<R, true> {
  using type = Cplx<R>;
  __device__ static inline void load(const type* p, R& re, R& im) {
    re = p->re;
    im = p->im;
  }
  __device__ static inline void store(type* p, R re, R im) {
    type v;
    v.re = re;
    v.im = im;
    *p = v;
  }
};

// One output element: D = op_D(alpha * acc + beta * op_C(C)), with the
// write-back modes of the reference (pack/writeback.rs:311-419): a plain store
// for alpha == 1, beta == 0; alpha scaling only when beta == 0 (C unread); the
// full form otherwise.
template <class R, bool CPLX>
__device__ inline void epilogue_store(const Epilogue& e, R acc_re, R acc_im, const typename Elem<R, CPLX>::type* c,
                                      typename Elem<R, CPLX>::type* d) {
  R vr, vi;
  if (e.plain) {
    vr = acc_re;
    vi = acc_im;
  } else {
    const R ar = (R)e.alpha_re, ai = (R)e.alpha_im;
    if (CPLX) {
      vr = acc_re * ar - acc_im * ai;
      vi = acc_re * ai + acc_im * ar;
    } else {
      vr = acc_re * ar;
      vi = R(0);
    }
    if (!e.beta_zero) {
      R cr, ci;
      Elem<R, CPLX>::load(c, cr, ci);
      if (e.conj_c) ci = -ci;
      const R br = (R)e.beta_re, bi = (R)e.beta_im;
      if (CPLX) {
        vr += cr * br - ci * bi;
        vi += cr * bi + ci * br;
      } else {
        vr += cr * br;
      }
    }
    if (CPLX && e.conj_d) vi = -vi;
  }
  Elem<R, CPLX>::store(d, vr, vi);
}

// Bounded wait on a nanosecond clock (the limit is per wait).
__device__ inline uint64_t globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

}  // namespace dev
}  // namespace tprims
