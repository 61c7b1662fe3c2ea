// Emulated FP64 products on the integer tensor cores (Ozaki scheme II); the
// kernels and their description are in ozaki.cu.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace evd {

constexpr int kOzMinMod = 4;     // fewest moduli (about 14-bit operands)
constexpr int kOzMaxMod = 16;    // most moduli (Mod < 2^126)
constexpr int kOzFp64Mod = 14;   // moduli for FP64-level products (53-bit operands)
constexpr long kOzMaxK = 65536;  // INT32 accumulation bound of the epilogue's reduction

// Byte offsets of the pieces of an emulated product's workspace.
struct OzLayout {
  long qa, qb, res, ea, eb, tr, bytes;
};

long oz_ld(long K);  // row pitch (bytes) of a quantised operand: K rounded up to 128
// 2-D tiled tensor map over `rows` rows of 16-bit elements (`elems` used of
// a row pitch of `ld` elements): boxes of 64 elements (128 bytes) x box_rows,
// 128-byte swizzle, zero fill outside the tensor.
int tma_map_rows16(CUtensorMap* map, const void* base, long rows, long elems, long ld,
                   int box_rows);
OzLayout oz_layout(long M, long N, long K, int nmod, bool need_transpose);
// bits P of the integer operands for nmod moduli and inner dimension K
int oz_bits(int nmod, long K);

// Rows of the operand = the `rows` columns of S (K long, column-major, lds):
// exponents into ex[rows], residues into Q (nmod planes of rows x oz_ld(K)).
int oz_quantize(long rows, long K, const double* S, long lds, int8_t* Q, int* ex, int nmod,
                cudaStream_t st);
// B = A^T (m x n column-major A)
int oz_transpose(long m, long n, const double* A, long lda, double* B, long ldb, cudaStream_t st);
// residue planes (M rounded up to 16) x N of (QA row m) . (QB row n) mod p_l
// lean: the 2-stage pipeline (130 KB of shared memory instead of 198 KB)
int oz_imma(long M, long N, long K, const int8_t* QA, const int8_t* QB, uint8_t* R, int nmod,
            bool lower, cudaStream_t st, bool lean = false);
// D = alpha 2^-(ea_m + eb_n) CRT(R) + beta C + diag I (lower: symmetric, mirrored)
int oz_crt(long M, long N, long K, const uint8_t* R, const int* ea, const int* eb, int nmod,
           double alpha, double beta, const double* C, long ldc, double diag, double* D, long ldd,
           bool lower, cudaStream_t st);
// the whole product: D = alpha op(A) op(B) + beta C + diag I
int oz_gemm(char ta, char tb, long M, long N, long K, double alpha, const double* A, long lda,
            const double* B, long ldb, double beta, const double* C, long ldc, double diag,
            double* D, long ldd, int nmod, bool lower, void* work, long lwork, cudaStream_t st,
            bool lean = false);
// C(lower, mirrored) = alpha (Y Z^T + Z Y^T) + beta C, Y and Z n x k
long oz_syr2k_ws_bytes(long n, long k, int nmod);
int oz_syr2k_lower(long n, long k, double alpha, const double* Y, long ldy, const double* Z,
                   long ldz, double beta, double* C, long ldc, int nmod, void* work, long lwork,
                   cudaStream_t st);
// reads (and clears) the error word of the tensor-core waits; synchronises st
int oz_check_err(cudaStream_t st);

// Emulated-product settings of a solve: moduli of the contractions and the
// workspace they use (nullptr / 0: FP64 DMMA products).
struct OzWork {
  int nmod;
  uint8_t* ws;
  long bytes;
};

}  // namespace evd
