// jit.cu — kernels given as expressions, compiled at run time (NVRTC).
//
// The reference takes the interaction kernel as a C++ std::function or a
// Python callable (include/fmma/fmma.hpp:65-87, cpython/pyfmma.cpp:150-151);
// neither can run on the device.  Here a caller passes f as a C++
// expression in x[q], y[q], dx[q] = x[q] - y[q], r2 = |x - y|^2, r = |x - y|.
// The kernel-dependent stages (M2L operator tables, per-pair M2L, near field,
// exact sum, nrnmm far field) are generated around the expression, compiled
// by NVRTC for sm_100a once per dimension at first use, loaded with the
// runtime's library API and launched through the same hook as a user
// __device__ functor; every other stage runs the library's own kernels.
// NVRTC is opened with dlopen, so the library has no link-time dependency
// on it.
#include <dlfcn.h>
#include <nvrtc.h>

#include <memory>
#include <mutex>
#include <string>

#include "fmma_internal.cuh"

namespace fmma_b200 {
namespace {

// Device code generated around the expression.  fmma_user_launch is restated
// field for field (same order and types as include/fmma_b200.h), so the
// launch record is passed to the kernels by value.
const char* kJitSource = R"JIT(
typedef long long i64;
typedef unsigned long long u64;
struct fmma_user_launch {
  int what, dim, nrhs;
  void* stream;
  double len;
  const double* node_all;
  int P, npad, kpad, noff;
  const int* offv;
  double* tab;
  i64 nrow;
  const int* row_box;
  const int* near;
  int nnear;
  const int *tb, *te, *sb, *se;
  const double* tx;
  i64 nt;
  const double* sx;
  i64 ns;
  const double* ws;
  const double* pot;
  const int* perm_t;
  void* out;
  int out_f32;
  const void* tgt;
  const void* src;
  const void* w;
  const i64* rows;
  const int* il;
  int nfar, level;
  const u64* key;
  const double* origin;
  double Len;
  const double* Wm;
  double* Wl;
  int grid_n, n;
  const double* gx;
  double* far;
};

__device__ __forceinline__ double fmma_f(const double* x, const double* y) {
  double dx[D_];
  double r2 = 0.0;
#pragma unroll
  for (int q = 0; q < D_; ++q) {
    dx[q] = x[q] - y[q];
    r2 += dx[q] * dx[q];
  }
  const double r = sqrt(r2);
  (void)r;
  return (double)(FMMA_EXPR);
}

__device__ void morton_decode_jit(u64 k, int bits, int* c) {
  for (int q = 0; q < D_; ++q) c[q] = 0;
  for (int b = 0; b < bits; ++b)
    for (int q = D_ - 1; q >= 0; --q) {
      c[q] |= (int)(k & 1ull) << b;
      k >>= 1;
    }
}

// tab[f][kl][km] = f(len * x_kl / 2, len * (o_f + x_km / 2))  (src/fmm_core.cpp:403-417)
extern "C" __global__ void jit_table(fmma_user_launch a) {
  const i64 total = (i64)a.noff * a.npad * a.kpad;
  for (i64 e = (i64)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (i64)gridDim.x * blockDim.x) {
    const i64 fo = e / ((i64)a.npad * a.kpad);
    const int rem = (int)(e - fo * a.npad * a.kpad);
    const int kl = rem / a.kpad, km = rem - kl * a.kpad;
    double v = 0.0;
    if (kl < a.P && km < a.P) {
      double x[D_], y[D_];
      for (int q = 0; q < D_; ++q) {
        x[q] = a.len * (a.node_all[kl * D_ + q] / 2);
        y[q] = a.len * ((double)a.offv[fo * 3 + q] + a.node_all[km * D_ + q] / 2);
      }
      v = fmma_f(x, y);
    }
    a.tab[e] = v;
  }
}

// near field, one thread per target  (src/fmm.cpp:121-141)
template <typename T>
__device__ void p2p_body(const fmma_user_launch& a) {
  for (i64 row = blockIdx.x; row < a.nrow; row += gridDim.x) {
    const int b = a.row_box[row];
    for (int t = a.tb[b] + threadIdx.x; t < a.te[b]; t += blockDim.x) {
      double x[D_];
      for (int q = 0; q < D_; ++q) x[q] = a.tx[(i64)q * a.nt + t];
      for (int r = 0; r < a.nrhs; ++r) {
        double acc = 0.0;
        for (int qn = 0; qn < a.nnear; ++qn) {
          const int s = a.near[row * a.nnear + qn];
          if (s < 0) continue;
          for (int j = a.sb[s]; j < a.se[s]; ++j) {
            double y[D_];
            for (int q = 0; q < D_; ++q) y[q] = a.sx[(i64)q * a.ns + j];
            acc += a.ws[(i64)r * a.ns + j] * fmma_f(x, y);
          }
        }
        const double v = acc + (a.pot ? a.pot[(i64)r * a.nt + t] : 0.0);
        static_cast<T*>(a.out)[(i64)r * a.nt + a.perm_t[t]] = (T)v;
      }
    }
  }
}
extern "C" __global__ void jit_p2p_d(fmma_user_launch a) { p2p_body<double>(a); }
extern "C" __global__ void jit_p2p_f(fmma_user_launch a) { p2p_body<float>(a); }

// direct sum  (src/fmma.cpp:80-94)
template <typename T>
__device__ void exact_body(const fmma_user_launch& a) {
  const T* tgt = static_cast<const T*>(a.tgt);
  const T* src = static_cast<const T*>(a.src);
  const T* w = static_cast<const T*>(a.w);
  for (i64 i = (i64)blockIdx.x * blockDim.x + threadIdx.x; i < a.nt; i += (i64)gridDim.x * blockDim.x) {
    const i64 ti = a.rows ? a.rows[i] : i;
    double x[D_];
    for (int q = 0; q < D_; ++q) x[q] = (double)tgt[ti * D_ + q];
    for (int r = 0; r < a.nrhs; ++r) {
      double acc = 0.0;
      for (i64 j = 0; j < a.ns; ++j) {
        double y[D_];
        for (int q = 0; q < D_; ++q) y[q] = (double)src[j * D_ + q];
        acc += (w ? (double)w[(i64)r * a.ns + j] : 1.0) * fmma_f(x, y);
      }
      static_cast<T*>(a.out)[(i64)r * a.nt + i] = (T)acc;
    }
  }
}
extern "C" __global__ void jit_exact_d(fmma_user_launch a) { exact_body<double>(a); }
extern "C" __global__ void jit_exact_f(fmma_user_launch a) { exact_body<float>(a); }

// M2L on absolute node coordinates  (src/fmm_core.cpp:456-492)
extern "C" __global__ void jit_m2l_pairwise(fmma_user_launch a, double o0, double o1, double o2) {
  const double origin[3] = {o0, o1, o2};
  const double len = a.Len / (double)(1 << a.level);
  for (i64 row = blockIdx.x; row < a.nrow; row += gridDim.x) {
    const int b = a.row_box[row];
    int cl[3] = {0, 0, 0};
    morton_decode_jit(a.key[b], a.level, cl);
    for (int kl = threadIdx.x; kl < a.P; kl += blockDim.x) {
      double x[D_];
      for (int q = 0; q < D_; ++q) x[q] = len * ((double)cl[q] + (1.0 + a.node_all[kl * D_ + q]) / 2) + origin[q];
      for (int r = 0; r < a.nrhs; ++r) {
        double acc = 0.0;
        for (int q = 0; q < a.nfar; ++q) {
          const int s = a.il[row * a.nfar + q];
          if (s < 0) continue;
          int cm[3] = {0, 0, 0};
          morton_decode_jit(a.key[s], a.level, cm);
          const double* wm = a.Wm + ((i64)s * a.nrhs + r) * a.kpad;
          for (int km = 0; km < a.P; ++km) {
            double y[D_];
            for (int qq = 0; qq < D_; ++qq)
              y[qq] = len * ((double)cm[qq] + (1.0 + a.node_all[km * D_ + qq]) / 2) + origin[qq];
            acc += fmma_f(x, y) * wm[km];
          }
        }
        a.Wl[((i64)b * a.nrhs + r) * a.kpad + kl] = acc;
      }
    }
  }
}

// nrnmm far field: boxes with sources not adjacent to the target's box
// (src/nrnmm.cpp:86-97)
extern "C" __global__ void jit_nrnmm_far(fmma_user_launch a) {
  i64 nbox = 1;
  for (int q = 0; q < D_; ++q) nbox *= a.grid_n;
  for (i64 t = (i64)blockIdx.x * blockDim.x + threadIdx.x; t < a.nt; t += (i64)gridDim.x * blockDim.x) {
    double x[D_];
    int bi[3] = {0, 0, 0};
    u64 kb = a.key[t];
    for (int q = D_ - 1; q >= 0; --q) {
      bi[q] = (int)(kb % (u64)a.grid_n);
      kb /= (u64)a.grid_n;
      x[q] = a.tx[(i64)q * a.nt + t];
    }
    for (int r = 0; r < a.nrhs; ++r) {
      double acc = 0.0;
      for (i64 s = 0; s < nbox; ++s) {
        if (a.se[s] <= a.sb[s]) continue;
        int si[3] = {0, 0, 0};
        i64 sc = s;
        bool near = true;
        for (int q = D_ - 1; q >= 0; --q) {
          si[q] = (int)(sc % a.grid_n);
          sc /= a.grid_n;
          near = near && (si[q] - bi[q] <= 1 && bi[q] - si[q] <= 1);
        }
        if (near) continue;
        const double* wm = a.Wm + (s * a.nrhs + r) * a.kpad;
        for (int k = 0; k < a.P; ++k) {
          double y[D_];
          int kc = k;
          for (int q = D_ - 1; q >= 0; --q) {
            y[q] = a.gx[((i64)q * a.grid_n + si[q]) * a.n + kc % a.n];
            kc /= a.n;
          }
          acc += fmma_f(x, y) * wm[k];
        }
      }
      a.far[(i64)r * a.nt + t] = acc;
    }
  }
}
)JIT";

struct Nvrtc {
  decltype(&nvrtcCreateProgram) create = nullptr;
  decltype(&nvrtcCompileProgram) compile = nullptr;
  decltype(&nvrtcGetProgramLogSize) log_size = nullptr;
  decltype(&nvrtcGetProgramLog) log = nullptr;
  decltype(&nvrtcGetCUBINSize) cubin_size = nullptr;
  decltype(&nvrtcGetCUBIN) cubin = nullptr;
  decltype(&nvrtcDestroyProgram) destroy = nullptr;
  bool ok = false;
};

const Nvrtc& nvrtc() {
  static Nvrtc n = [] {
    Nvrtc r;
    void* h = dlopen("libnvrtc.so.12", RTLD_NOW | RTLD_LOCAL);
    if (!h) h = dlopen("/usr/local/cuda/lib64/libnvrtc.so.12", RTLD_NOW | RTLD_LOCAL);
    if (!h) h = dlopen("libnvrtc.so", RTLD_NOW | RTLD_LOCAL);
    if (!h) return r;
    r.create = (decltype(r.create))dlsym(h, "nvrtcCreateProgram");
    r.compile = (decltype(r.compile))dlsym(h, "nvrtcCompileProgram");
    r.log_size = (decltype(r.log_size))dlsym(h, "nvrtcGetProgramLogSize");
    r.log = (decltype(r.log))dlsym(h, "nvrtcGetProgramLog");
    r.cubin_size = (decltype(r.cubin_size))dlsym(h, "nvrtcGetCUBINSize");
    r.cubin = (decltype(r.cubin))dlsym(h, "nvrtcGetCUBIN");
    r.destroy = (decltype(r.destroy))dlsym(h, "nvrtcDestroyProgram");
    r.ok = r.create && r.compile && r.log_size && r.log && r.cubin_size && r.cubin && r.destroy;
    return r;
  }();
  return n;
}

struct JitModule {
  bool built = false;
  cudaLibrary_t lib = nullptr;
  cudaKernel_t table = nullptr, p2p_d = nullptr, p2p_f = nullptr, exact_d = nullptr, exact_f = nullptr,
               pairwise = nullptr, nrnmm_far = nullptr;
};

struct JitKernel {
  std::string expr;
  std::mutex mu;
  JitModule mod[4];  // by dimension
  ~JitKernel() {
    for (auto& m : mod)
      if (m.lib) cudaLibraryUnload(m.lib);
  }
};

// Compiles the stages for one dimension; throws with the compiler's log.
void build_module(JitKernel& jk, int dim) {
  JitModule& m = jk.mod[dim];
  if (m.built) return;
  const Nvrtc& nv = nvrtc();
  if (!nv.ok) throw Error(FMMA_ERR_NO_DEVICE, "kernel expressions need NVRTC (libnvrtc.so.12), which is not available");
  const std::string src = "#define D_ " + std::to_string(dim) + "\n#define FMMA_EXPR (" + jk.expr + ")\n" + kJitSource;
  nvrtcProgram prog;
  if (nv.create(&prog, src.c_str(), "fmma_expr.cu", 0, nullptr, nullptr) != NVRTC_SUCCESS)
    throw Error(FMMA_ERR_CUDA, "nvrtcCreateProgram failed");
  const char* opts[] = {"--gpu-architecture=sm_100a", "--std=c++17", "-default-device"};
  const nvrtcResult rc = nv.compile(prog, 3, opts);
  if (rc != NVRTC_SUCCESS) {
    size_t n = 0;
    nv.log_size(prog, &n);
    std::string log(n, '\0');
    if (n) nv.log(prog, &log[0]);
    nv.destroy(&prog);
    throw Error(FMMA_ERR_INVALID_ARG, "kernel expression does not compile: " + log);
  }
  size_t nbin = 0;
  nv.cubin_size(prog, &nbin);
  std::string bin(nbin, '\0');
  nv.cubin(prog, &bin[0]);
  nv.destroy(&prog);
  FMMA_CHECK_CUDA(cudaLibraryLoadData(&m.lib, bin.data(), nullptr, nullptr, 0, nullptr, nullptr, 0));
  FMMA_CHECK_CUDA(cudaLibraryGetKernel(&m.table, m.lib, "jit_table"));
  FMMA_CHECK_CUDA(cudaLibraryGetKernel(&m.p2p_d, m.lib, "jit_p2p_d"));
  FMMA_CHECK_CUDA(cudaLibraryGetKernel(&m.p2p_f, m.lib, "jit_p2p_f"));
  FMMA_CHECK_CUDA(cudaLibraryGetKernel(&m.exact_d, m.lib, "jit_exact_d"));
  FMMA_CHECK_CUDA(cudaLibraryGetKernel(&m.exact_f, m.lib, "jit_exact_f"));
  FMMA_CHECK_CUDA(cudaLibraryGetKernel(&m.pairwise, m.lib, "jit_m2l_pairwise"));
  FMMA_CHECK_CUDA(cudaLibraryGetKernel(&m.nrnmm_far, m.lib, "jit_nrnmm_far"));
  m.built = true;
}

int launch(cudaKernel_t k, unsigned grid, unsigned block, void** args, cudaStream_t st) {
  return (int)cudaLaunchKernel((const void*)k, dim3(grid < 1 ? 1 : grid), dim3(block), args, 0, st);
}

// The hook the library calls for the kernel-dependent stages.
int jit_hook(const fmma_user_launch* a, void* user) {
  JitKernel& jk = *static_cast<JitKernel*>(user);
  if (a->dim < 1 || a->dim > 3) return (int)cudaErrorInvalidValue;
  {
    std::lock_guard<std::mutex> lk(jk.mu);
    try {
      build_module(jk, a->dim);
    } catch (const Error& e) {
      set_last_error(e.what());
      return (int)cudaErrorInvalidSource;
    }
  }
  const JitModule& m = jk.mod[a->dim];
  cudaStream_t st = static_cast<cudaStream_t>(a->stream);
  fmma_user_launch rec = *a;
  void* args1[] = {&rec};
  switch (a->what) {
    case FMMA_USER_TABLE: {
      const long long total = (long long)a->noff * a->npad * a->kpad;
      const long long g = std::min<long long>((total + 255) / 256, 148 * 32);
      return launch(m.table, (unsigned)g, 256, args1, st);
    }
    case FMMA_USER_P2P:
      return launch(a->out_f32 ? m.p2p_f : m.p2p_d, (unsigned)std::min<long long>(a->nrow, 148 * 64), 128, args1, st);
    case FMMA_USER_EXACT:
      return launch(a->out_f32 ? m.exact_f : m.exact_d, (unsigned)((a->nt + 127) / 128), 128, args1, st);
    case FMMA_USER_M2L_PAIRWISE: {
      double o[3] = {0.0, 0.0, 0.0};
      for (int q = 0; q < a->dim; ++q) o[q] = a->origin[q];
      void* args[] = {&rec, &o[0], &o[1], &o[2]};
      return launch(m.pairwise, (unsigned)std::min<long long>(a->nrow, 148 * 16), 128, args, st);
    }
    case FMMA_USER_NRNMM_FAR:
      return launch(m.nrnmm_far, (unsigned)((a->nt + 127) / 128), 128, args1, st);
    default:
      return (int)cudaErrorInvalidValue;
  }
}

}  // namespace

// Installs an expression kernel on the context (see fmma_set_kernel_expr).
void set_kernel_expr(fmma_ctx* ctx, const char* expr, int translation_invariant) {
  FMMA_REQUIRE(expr != nullptr && expr[0] != '\0', "empty kernel expression");
  auto jk = std::make_shared<JitKernel>();
  jk->expr = expr;
  FMMA_CHECK_CUDA(cudaSetDevice(ctx->device));
  build_module(*jk, 3);  // reject an expression that does not compile now, not at the first solve
  ctx->user_own = jk;
  ctx->user_hook = &jit_hook;
  ctx->user_ptr = jk.get();
  ctx->user_ti = translation_invariant ? 1 : 0;
  ctx->kernel_id = kUserKernel;
  ctx->user_gen++;
}

}  // namespace fmma_b200
