// fmma/device.cuh — user __device__ functors for fmma::FMMA (nvcc only).
//
//   #include "fmma/device.cuh"
//   struct MyKernel {
//     __device__ double operator()(const std::array<double, 2>& x,
//                                  const std::array<double, 2>& y) const { ... }
//   };
//   fmma::FMMA<double, 2> f;
//   f.set_fn_device(MyKernel{});            // or an extended __device__ lambda
//
// Replaces set_fn with an arbitrary functor (reference include/fmma/fmma.hpp:
// 65-87).  The kernel-dependent stages (M2L operator tables, per-pair M2L,
// P2P, exact, nrnmm far field) are instantiated here, in the caller's translation unit, and
// launched by libfmma_b200 through a hook (fmma_set_user_kernel); all other
// stages run inside the library.  Compile with --expt-relaxed-constexpr
// (std::array in device code) and -gencode arch=compute_100a,code=sm_100a.
#pragma once

#include <cuda_runtime.h>

#include <array>
#include <memory>

#include "fmma.hpp"

namespace fmma {
namespace gpu {

template <int D>
using dpoint = std::array<double, D>;

__device__ __forceinline__ void morton_decode_dev(uint64_t k, int dim, int bits, int* c) {
  for (int q = 0; q < dim; ++q) c[q] = 0;
  for (int b = 0; b < bits; ++b)
    for (int q = dim - 1; q >= 0; --q) {
      c[q] |= (int)(k & 1) << b;
      k >>= 1;
    }
}

// tab[f][kl][km] = f(len * x_kl / 2, len * (o_f + x_km / 2)) (src/fmm_core.cpp:403-417)
template <class F, int D>
__global__ void k_user_table(F f, double len, const double* node_all, int P, int npad, int kpad, int noff,
                             const int* offv, double* tab) {
  const long long total = (long long)noff * npad * kpad;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
    const long long fo = e / ((long long)npad * kpad);
    const int rem = (int)(e - fo * npad * kpad);
    const int kl = rem / kpad, km = rem - kl * kpad;
    double v = 0.0;
    if (kl < P && km < P) {
      dpoint<D> x, y;
      for (int q = 0; q < D; ++q) {
        x[q] = len * (node_all[kl * D + q] / 2);
        y[q] = len * ((double)offv[fo * 3 + q] + node_all[km * D + q] / 2);
      }
      v = f(x, y);
    }
    tab[e] = v;
  }
}

// Near field, one thread per target (src/fmm.cpp:121-141).
template <class F, int D, typename T>
__global__ void k_user_p2p(F f, fmma_user_launch a) {
  for (long long row = blockIdx.x; row < a.nrow; row += gridDim.x) {
    const int b = a.row_box[row];
    for (int t = a.tb[b] + threadIdx.x; t < a.te[b]; t += blockDim.x) {
      dpoint<D> x;
      for (int q = 0; q < D; ++q) x[q] = a.tx[(long long)q * a.nt + t];
      for (int r = 0; r < a.nrhs; ++r) {
        double acc = 0.0;
        for (int qn = 0; qn < a.nnear; ++qn) {
          const int s = a.near[row * a.nnear + qn];
          if (s < 0) continue;
          for (int j = a.sb[s]; j < a.se[s]; ++j) {
            dpoint<D> y;
            for (int q = 0; q < D; ++q) y[q] = a.sx[(long long)q * a.ns + j];
            acc += a.ws[(long long)r * a.ns + j] * f(x, y);
          }
        }
        const double v = acc + (a.pot ? a.pot[(long long)r * a.nt + t] : 0.0);
        static_cast<T*>(a.out)[(long long)r * a.nt + a.perm_t[t]] = (T)v;
      }
    }
  }
}

// Direct sum (src/fmma.cpp:80-101).
template <class F, int D, typename T>
__global__ void k_user_exact(F f, fmma_user_launch a) {
  const T* tgt = static_cast<const T*>(a.tgt);
  const T* src = static_cast<const T*>(a.src);
  const T* w = static_cast<const T*>(a.w);
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < a.nt; i += (long long)gridDim.x * blockDim.x) {
    const long long ti = a.rows ? a.rows[i] : i;
    dpoint<D> x;
    for (int q = 0; q < D; ++q) x[q] = (double)tgt[ti * D + q];
    for (int r = 0; r < a.nrhs; ++r) {
      double acc = 0.0;
      for (long long j = 0; j < a.ns; ++j) {
        dpoint<D> y;
        for (int q = 0; q < D; ++q) y[q] = (double)src[j * D + q];
        acc += (w ? (double)w[(long long)r * a.ns + j] : 1.0) * f(x, y);
      }
      static_cast<T*>(a.out)[(long long)r * a.nt + i] = (T)acc;
    }
  }
}

// M2L on absolute node coordinates (src/fmm_core.cpp:456-492).
template <class F, int D>
__global__ void k_user_m2l_pairwise(F f, fmma_user_launch a, dpoint<D> origin) {
  const double len = a.Len / (double)(1 << a.level);
  for (long long row = blockIdx.x; row < a.nrow; row += gridDim.x) {
    const int b = a.row_box[row];
    int cl[3] = {0, 0, 0};
    morton_decode_dev(a.key[b], D, a.level, cl);
    for (int kl = threadIdx.x; kl < a.P; kl += blockDim.x) {
      dpoint<D> x;
      for (int q = 0; q < D; ++q) x[q] = len * ((double)cl[q] + (1.0 + a.node_all[kl * D + q]) / 2) + origin[q];
      for (int r = 0; r < a.nrhs; ++r) {
        double acc = 0.0;
        for (int q = 0; q < a.nfar; ++q) {
          const int s = a.il[row * a.nfar + q];
          if (s < 0) continue;
          int cm[3] = {0, 0, 0};
          morton_decode_dev(a.key[s], D, a.level, cm);
          const double* wm = a.Wm + ((long long)s * a.nrhs + r) * a.kpad;
          for (int km = 0; km < a.P; ++km) {
            dpoint<D> y;
            for (int qq = 0; qq < D; ++qq)
              y[qq] = len * ((double)cm[qq] + (1.0 + a.node_all[km * D + qq]) / 2) + origin[qq];
            acc += f(x, y) * wm[km];
          }
        }
        a.Wl[((long long)b * a.nrhs + r) * a.kpad + kl] = acc;
      }
    }
  }
}

// nrnmm far field: every box with sources that is not adjacent to the
// target's box, through its Chebyshev nodes (src/nrnmm.cpp:86-97).
template <class F, int D>
__global__ void k_user_nrnmm_far(F f, fmma_user_launch a) {
  long long nbox = 1;
  for (int q = 0; q < D; ++q) nbox *= a.grid_n;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < a.nt; t += (long long)gridDim.x * blockDim.x) {
    dpoint<D> x;
    int bi[3] = {0, 0, 0};
    unsigned long long kb = a.key[t];
    for (int q = D - 1; q >= 0; --q) {
      bi[q] = (int)(kb % (unsigned long long)a.grid_n);
      kb /= (unsigned long long)a.grid_n;
      x[q] = a.tx[(long long)q * a.nt + t];
    }
    for (int r = 0; r < a.nrhs; ++r) {
      double acc = 0.0;
      for (long long s = 0; s < nbox; ++s) {
        if (a.se[s] <= a.sb[s]) continue;
        int si[3] = {0, 0, 0};
        long long sc = s;
        bool near = true;
        for (int q = D - 1; q >= 0; --q) {
          si[q] = (int)(sc % a.grid_n);
          sc /= a.grid_n;
          near = near && (si[q] - bi[q] <= 1 && bi[q] - si[q] <= 1);
        }
        if (near) continue;
        const double* wm = a.Wm + (s * a.nrhs + r) * a.kpad;
        for (int k = 0; k < a.P; ++k) {
          dpoint<D> y;
          int kc = k;
          for (int q = D - 1; q >= 0; --q) {
            y[q] = a.gx[((long long)q * a.grid_n + si[q]) * a.n + kc % a.n];
            kc /= a.n;
          }
          acc += f(x, y) * wm[k];
        }
      }
      a.far[(long long)r * a.nt + t] = acc;
    }
  }
}

template <class F, int D>
int user_hook(const fmma_user_launch* a, void* user) {
  const F& f = *static_cast<const F*>(user);
  cudaStream_t s = static_cast<cudaStream_t>(a->stream);
  switch (a->what) {
    case FMMA_USER_TABLE: {
      long long total = (long long)a->noff * a->npad * a->kpad;
      int g = (int)((total + 255) / 256);
      if (g > 148 * 32) g = 148 * 32;
      k_user_table<F, D><<<g < 1 ? 1 : g, 256, 0, s>>>(f, a->len, a->node_all, a->P, a->npad, a->kpad, a->noff,
                                                        a->offv, a->tab);
      break;
    }
    case FMMA_USER_P2P: {
      int g = (int)(a->nrow < 148 * 64 ? a->nrow : 148 * 64);
      if (a->out_f32) k_user_p2p<F, D, float><<<g < 1 ? 1 : g, 128, 0, s>>>(f, *a);
      else k_user_p2p<F, D, double><<<g < 1 ? 1 : g, 128, 0, s>>>(f, *a);
      break;
    }
    case FMMA_USER_EXACT: {
      int g = (int)((a->nt + 127) / 128);
      if (a->out_f32) k_user_exact<F, D, float><<<g < 1 ? 1 : g, 128, 0, s>>>(f, *a);
      else k_user_exact<F, D, double><<<g < 1 ? 1 : g, 128, 0, s>>>(f, *a);
      break;
    }
    case FMMA_USER_M2L_PAIRWISE: {
      dpoint<D> o;
      for (int q = 0; q < D; ++q) o[q] = a->origin[q];
      int g = (int)(a->nrow < 148 * 16 ? a->nrow : 148 * 16);
      k_user_m2l_pairwise<F, D><<<g < 1 ? 1 : g, 128, 0, s>>>(f, *a, o);
      break;
    }
    case FMMA_USER_NRNMM_FAR: {
      int g = (int)((a->nt + 127) / 128);
      k_user_nrnmm_far<F, D><<<g < 1 ? 1 : g, 128, 0, s>>>(f, *a);
      break;
    }
    default:
      return (int)cudaErrorInvalidValue;
  }
  return (int)cudaGetLastError();
}

}  // namespace gpu

template <typename TYPE, std::size_t DIM>
template <class F>
void FMMA<TYPE, DIM>::set_fn_device(F f, bool translation_invariant) {
  user_obj_ = std::shared_ptr<void>(new F(f), [](void* p) { delete static_cast<F*>(p); });
  user_hook_ = &gpu::user_hook<F, (int)DIM>;
  user_ti_ = translation_invariant;
  expr_ = false;
}

}  // namespace fmma
