// Internal interface of the panel factorisation (panel_qr.cu).
#pragma once
#include <cuda_runtime.h>

namespace evd {

// Doubles of workspace for an m x 32 panel (stacked R factors, node Q blocks,
// arrival counters).
long panel_qr_ws_doubles(long m);
int panel_qr_check(long m, long n, long lda);
// Zero the arrival counters for panels of up to m rows (needed once per
// workspace; the kernels reset each counter after use).
int panel_counters_reset(long m, double* ws, cudaStream_t st);
// mode 0: A <- explicit thin Q.  mode 1: Yout <- Y, Wout <- W, R <- R and, if
// Aband != nullptr, the panel of the band matrix (R over zeros) into Aband.
int panel_qr_launch(long m, double* A, long lda, double* ws, int mode, double* Yout, long ldy,
                    double* Wout, long ldw, double* R, long ldr, double* Aband, long ldband,
                    cudaStream_t st);

}  // namespace evd
