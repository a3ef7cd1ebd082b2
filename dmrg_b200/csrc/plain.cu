// The per-block matvec schedule: one library GEMM per task row, in task order,
// exactly the loop of the reference's av() (src/core.cpp:22-31 ->
// qtensor::contract(T*, T*, map, ...) src/qtensor.cpp:986-994 ->
// tensor::contract src/tensor.cpp:698-718 -> dgemm/zgemm src/dgemm.cpp:29-47),
// on the GPU.  It is the plain FP64 path the grouped kernels are measured
// against.  Row-major C[M x N] += sign A[M x K] B[N x K]^T is the column-major
// call C^T = B A^T: gemm(T, N, N, M, K, sign, B, K, A, K, 1, C, N).
// cuBLAS is loaded at run time (libcublas.so.12).
#include <cublas_v2.h>
#include <cuda_runtime.h>
#include <dlfcn.h>

#include <cstdlib>
#include <mutex>
#include <string>

#include "../../include/dmrgx.h"
#include "ctx.h"

namespace dmrgx {
namespace {

struct Blas {
  bool tried = false, ok = false;
  decltype(&cublasCreate_v2) create;
  decltype(&cublasDestroy_v2) destroy;
  decltype(&cublasSetStream_v2) set_stream;
  decltype(&cublasDgemm_v2) dgemm;
  decltype(&cublasZgemm_v2) zgemm;
};
Blas g_blas;
std::mutex g_blas_mu;

bool load_blas() {
  std::lock_guard<std::mutex> lk(g_blas_mu);
  if (g_blas.tried) return g_blas.ok;
  g_blas.tried = true;
  const char* names[] = {getenv("DMRGX_CUBLAS"), "libcublas.so.12",
                         "/usr/local/cuda/lib64/libcublas.so.12", "libcublas.so"};
  void* lib = nullptr;
  for (const char* n : names)
    if (n && (lib = dlopen(n, RTLD_NOW | RTLD_LOCAL))) break;
  if (!lib) return false;
#define SYM(field, name)                                    \
  g_blas.field = (decltype(g_blas.field))dlsym(lib, #name); \
  if (!g_blas.field) return false;
  SYM(create, cublasCreate_v2);
  SYM(destroy, cublasDestroy_v2);
  SYM(set_stream, cublasSetStream_v2);
  SYM(dgemm, cublasDgemm_v2);
  SYM(zgemm, cublasZgemm_v2);
#undef SYM
  g_blas.ok = true;
  return true;
}

int stage(dmrgx_ctx* c, cublasHandle_t h, const std::vector<PlainRow>& rows, const double* A,
          const double* B, double* C, int64_t c_len) {
  const bool cplx = c->dtype == DMRGX_C128;
  if (cudaMemsetAsync(C, 0, sizeof(double) * c_len, c->stream) != cudaSuccess) return DMRGX_E_CUDA;
  for (const PlainRow& r : rows) {
    cublasStatus_t st;
    if (cplx) {
      const cuDoubleComplex al = make_cuDoubleComplex((double)r.sign, 0.0),
                            be = make_cuDoubleComplex(1.0, 0.0);
      st = g_blas.zgemm(h, CUBLAS_OP_T, CUBLAS_OP_N, r.N, r.M, r.K, &al,
                        (const cuDoubleComplex*)(B + r.b_off), r.K,
                        (const cuDoubleComplex*)(A + r.a_off), r.K, &be,
                        (cuDoubleComplex*)(C + r.c_off), r.N);
    } else {
      const double al = (double)r.sign, be = 1.0;
      st = g_blas.dgemm(h, CUBLAS_OP_T, CUBLAS_OP_N, r.N, r.M, r.K, &al, B + r.b_off, r.K,
                        A + r.a_off, r.K, &be, C + r.c_off, r.N);
    }
    if (st != CUBLAS_STATUS_SUCCESS) {
      set_error("per-block matvec: cuBLAS GEMM failed");
      return DMRGX_E_CUDA;
    }
  }
  return 0;
}

}  // namespace

int run_matvec_plain(dmrgx_ctx* c, const double* in, double* out) {
  if (!c->blas) {
    if (!load_blas()) {
      set_error("per-block matvec: cuBLAS (libcublas.so.12) could not be loaded");
      return DMRGX_E_CUDA;
    }
    cublasHandle_t h = nullptr;
    if (g_blas.create(&h) != CUBLAS_STATUS_SUCCESS) {
      set_error("per-block matvec: cuBLAS initialisation failed");
      return DMRGX_E_CUDA;
    }
    c->blas = h;
  }
  cublasHandle_t h = (cublasHandle_t)c->blas;
  g_blas.set_stream(h, c->stream);
  const int f = c->f();
  c->prof_mark();
  c->prof_mark();
  double* store = (double*)c->store.p;
  int rc = stage(c, h, c->st1.rows, (const double*)c->renv.p, in, store, c->d_store * f);
  c->prof_mark();
  if (!rc) rc = stage(c, h, c->st2.rows, (const double*)c->lenv.p, store, out, c->n * f);
  c->prof_mark();
  return rc;
}

void plain_release(dmrgx_ctx* c) {
  if (c->blas && g_blas.ok) g_blas.destroy((cublasHandle_t)c->blas);
  c->blas = nullptr;
}

}  // namespace dmrgx
