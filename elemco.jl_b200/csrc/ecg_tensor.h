// ecg_tensor.h — device workspace arena and the tensor-contraction helper.
//
// contract() evaluates  C[ic] = alpha * sum A[ia] B[ib] + beta * C[ic]  for
// dense column-major device tensors named by single-character index strings
// (first character = fastest index), the way TensorOperations' @tensor does
// in the reference (src/tools/tensortools.jl:38-45): operands that are not
// already in a GEMM-compatible order are permuted into workspace, one FP64
// GEMM runs, and the result is permuted back if needed.  Among the index
// orders that make A, B or C directly usable, the one that copies the fewest
// elements is chosen.
#pragma once
#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

#include "ecg_dev.h"

namespace ecg {

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

// Bump allocator over one device buffer; release() returns to a mark.
class Arena {
 public:
  void init(double* base, int64_t cap) {
    base_ = base;
    cap_ = cap;
    top_ = 0;
    peak_ = 0;
  }
  double* get(int64_t n);
  int64_t mark() const { return top_; }
  void release(int64_t m) { top_ = m; }
  int64_t peak() const { return peak_; }
  int64_t capacity() const { return cap_; }

 private:
  double* base_ = nullptr;
  int64_t cap_ = 0, top_ = 0, peak_ = 0;
};

// Extent of an index character for the current system.
struct Extents {
  int64_t no = 0, nv = 0, nq = 0, n = 0;
  int64_t operator()(char c) const;
};

// FP64 GEMM, or — when `mixed` and the product has at least 2^26 multiply-adds —
// the split-BF16 tensor-core GEMM (FP32-level accuracy).
int gemm_prec(bool mixed, dev::stream_t s, char ta, char tb, int64_t m, int64_t n, int64_t k,
              double alpha, const double* A, int64_t lda, const double* B, int64_t ldb,
              double beta, double* C, int64_t ldc);

class Contractor {
 public:
  Contractor(dev::stream_t s, Arena* ws, const Extents* ext, bool mixed = false)
      : s_(s), ws_(ws), ext_(ext), mixed_(mixed) {}
  void operator()(double alpha, const double* A, const char* ia, const double* B,
                  const char* ib, double beta, double* C, const char* ic);
  // out[io] = alpha * in[ii] + beta * out[io]   (pure permutation)
  void permute(double alpha, const double* in, const char* ii, double beta, double* out,
               const char* io);
  int64_t size(const char* idx) const;

 private:
  dev::stream_t s_;
  Arena* ws_;
  const Extents* ext_;
  bool mixed_;
};

void check(int code, const char* what);

}  // namespace ecg
