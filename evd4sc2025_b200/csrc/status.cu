// Status strings and version of the C ABI.
#include "common.cuh"

extern "C" const char* evd_status_string(int status) {
  switch (status) {
    case EVD_SUCCESS: return "success";
    case EVD_ERR_INVALID_ARG: return "invalid argument";
    case EVD_ERR_CUDA: return "CUDA runtime error";
    case EVD_ERR_TIMEOUT: return "bounded device wait timed out";
    case EVD_ERR_NO_CONVERGENCE: return "iteration did not converge";
    case EVD_ERR_WORKSPACE: return "workspace too small";
    default: return "unknown status";
  }
}

extern "C" const char* evd_version(void) { return "evd_b200 0.1 sm_100a"; }
