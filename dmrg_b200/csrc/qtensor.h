// Device block-sparse tensors for the site step around the matvec: the
// environment (x) MPO fusion, the permutes, the environment update and the
// SVD truncation.  Metadata (sector sizes, block labels, fermion directions,
// block order) lives on the host and follows the reference's qtensor
// bookkeeping exactly (include/qtensor.h:20-223, src/qtensor.cpp); the values
// live in one device buffer per tensor, blocks packed in block order, each block
// row-major (last index fastest).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <string>
#include <vector>

#include "grouped.h"
#include "qmeta.h"

namespace dmrgx {

struct QTensor {
  QMeta m;
  std::vector<int64_t> off;  // element offset of every block (+ total at the end)
  double* d = nullptr;       // device values, f doubles per element
  int f = 1;                 // 1 real, 2 complex (interleaved)
  cudaStream_t st = nullptr; // stream the values were allocated on (freed there)
  QTensor() = default;
  QTensor(const QTensor&) = delete;
  QTensor& operator=(const QTensor&) = delete;
  ~QTensor();
  int64_t total() const { return off.empty() ? 0 : off.back(); }
  int64_t bsize(int b) const { return off[b + 1] - off[b]; }
  // (re)compute offsets from the metadata and allocate zeroed device values
  cudaError_t alloc(cudaStream_t s);
};
using QTPtr = std::shared_ptr<QTensor>;

// Element-wise gather: dst block elements at multi-index idx (dims, last
// fastest) receive sum over sources of sign * src[src_off + idx . strides]
// (conj: complex conjugate), written at dst_off + idx . dst_strides.
struct GOut {
  int64_t dst_off, size;
  int32_t rank, src_begin, src_count, pad_;
  int32_t dims[8];
  int64_t dst_strides[8];
};
struct GSrc {
  int64_t src_off;
  int64_t strides[8];
  double sign;
  int32_t conj, pad_;
};

cudaError_t launch_gather(const double* src, double* dst, const std::vector<GOut>& outs,
                          const std::vector<GSrc>& srcs, bool cplx, cudaStream_t st);

// The context-independent engine state (stream, group rule, SVD library handle).
struct Engine {
  cudaStream_t stream = nullptr;
  int device = 0;
  int num_sms = 148;
  Group G;
  int f = 1;
};

// Block pairs of the reference's contract(A, a, B, b, change, fermion)
// (src/qtensor.cpp:902-983) with their fermion signs; sym = output labels before
// any exchange (legs A[0..a), B[0..b), B(b..], A(a..]).
struct FusePair {
  int l, r;
  double sign;
  std::vector<int> sym;
};
std::vector<FusePair> fuse_pairs(const Group& G, const QMeta& A, int a, const QMeta& B, int b,
                                 bool change);

// C_o = sum_s A_s B_s^T over grouped descriptors (FP64 / complex, see grouped.h);
// synchronous on E.stream
cudaError_t qt_grouped_gemm(const Engine& E, const double* A, const double* B, double* C,
                            std::vector<DOut>& outs, std::vector<DSeg>& segs);

QTPtr qt_from_host(const Engine& E, const int* meta, const void* vals, std::string& err);
int qt_to_host(const QTensor& T, std::vector<int>& meta, std::vector<double>& vals,
               cudaStream_t s);
QTPtr qt_copy(const Engine& E, const QTensor& A);

// reference qtensor::contract(A, a, B, b, change, fermion) (src/qtensor.cpp:902-983)
// followed by exchange(x, y) when x != y (src/qtensor.cpp:349-373): the env (x)
// MPO fusion of src/core.cpp:188-192.
QTPtr qt_contract_legs(const Engine& E, const QTensor& A, int a, const QTensor& B, int b,
                       bool change, int ex0, int ex1, std::string& err);
// reference qtensor::exchange(a, b) alone
QTPtr qt_exchange(const Engine& E, const QTensor& A, int a, int b, std::string& err);
// reference qtensor::contract(A, B, transa, transb, num) (src/qtensor.cpp:824-899)
QTPtr qt_contract_mat(const Engine& E, const QTensor& A, const QTensor& B, char ta, char tb,
                      int num, std::string& err);
// reference qtensor::conjugate() (src/qtensor.cpp:297-303), in place
int qt_conjugate(const Engine& E, QTensor& A);
// reference qtensor::svd(U, S, V, num, cutoff) (src/qtensor.cpp:1122-1262): U, V and
// the singular values sorted as the reference sorts them
int qt_svd(const Engine& E, const QTensor& A, int num, int cutoff, QTPtr& U, QTPtr& V,
           std::vector<double>& s, std::string& err);

}  // namespace dmrgx
