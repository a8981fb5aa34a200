// jg_noalloc.cu -- block point relaxation that allocates no memory.
//
// Some hosts cannot call cudaMalloc at the point where they want a linear
// solve: their device memory belongs to another allocator (a framework pool
// that claimed the GPU's memory up front, or an embedding application that
// budgets every byte), or they cannot afford an allocation's implicit device
// synchronisation or an out-of-memory failure in the middle of a run.  The
// regular entry points allocate their working memory in jg_create; this one
// works on buffers the caller already owns.
//
// jg_relax_csr_noalloc runs block Jacobi sweeps on a system given in the
// reference's own layout (CSR over nbocv, diagonal block first, A[nnz][5][5],
// rhs/dq[ncv][5]) -- the iteration of jg_solve_lin_sys with lin_solver =
// JG_LS_JACOBI, agreeing with it to rounding (here each sweep solves with the
// LU factors, as lusolv does; that path multiplies by the stored inverse).
// Its only working memory is one vector of
// JG_NOALLOC_MAX_CELLS x 5 doubles (2.5 MiB) in a file-scope __device__ array,
// which every GPU that loads the library holds until the process exits.
#include <cuda_runtime.h>

#include <atomic>
#include <cstdio>
#include <mutex>

#include "jg_internal.h"

// Ping-pong partner of the caller's dq during the sweeps.  Shared by every call
// on a device: calls that overlap on the GPU (other streams, other threads)
// race on it.  Nothing in it needs to start at zero: the first sweep never
// reads it.
static __device__ __align__(256) double g_relax_scratch[JG_NOALLOC_MAX_CELLS * 5];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
std::atomic<double*> g_scratch_ptr[kMaxDevices];  // device address of g_relax_scratch, per device

// The host-side name g_relax_scratch is only a stand-in for the device symbol;
// the kernel needs its device address, looked up once per device with that
// device current.
int scratch_address(int dev, double** out) {
  if (dev < 0 || dev >= kMaxDevices) return JG_ERR_ARG;
  double* p = g_scratch_ptr[dev].load();
  if (p) {
    *out = p;
    return JG_OK;
  }
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  p = g_scratch_ptr[dev].load();
  if (!p) {
    void* addr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&addr, g_relax_scratch);
    if (e != cudaSuccess || addr == nullptr) return JG_ERR_CUDA;
    p = (double*)addr;
    g_scratch_ptr[dev].store(p);
  }
  *out = p;
  return JG_OK;
}

// LU of the 5x5 diagonal block without pivoting and the forward/back
// substitution, as the reference's ludeco / lusolv (UgpWithCv.cpp:2489-2543)
__device__ void lu_solve5(double* A, double* c) {
  for (int jc = 1; jc < 5; jc++) A[jc] /= A[0];
  for (int jrjc = 1;; jrjc++) {
    for (int jr = jrjc; jr < 5; jr++) {
      double sum = A[5 * jr + jrjc];
      for (int jm = 0; jm < jrjc; jm++) sum -= A[5 * jr + jm] * A[5 * jm + jrjc];
      A[5 * jr + jrjc] = sum;
    }
    if (jrjc == 4) break;
    for (int jc = jrjc + 1; jc < 5; jc++) {
      double sum = A[5 * jrjc + jc];
      for (int jm = 0; jm < jrjc; jm++) sum -= A[5 * jrjc + jm] * A[5 * jm + jc];
      A[5 * jrjc + jc] = sum / A[5 * jrjc + jrjc];
    }
  }
  c[0] = c[0] / A[0];
  for (int jr = 1; jr < 5; jr++) {
    double sum = c[jr];
    for (int jm = 0; jm < jr; jm++) sum -= A[5 * jr + jm] * c[jm];
    c[jr] = sum / A[5 * jr + jr];
  }
  for (int jr = 3; jr >= 0; jr--) {  // lusolv subtracts from the last column back
    double sum = c[jr];
    for (int jm = 4; jm > jr; jm--) sum -= A[5 * jr + jm] * c[jm];
    c[jr] = sum;
  }
}

// One Jacobi sweep over CSR rows: x_out[c] = D_c^-1 (rhs_c - sum_k A_k x_in[nb_k]);
// on the first sweep x_in = 0 and is not read.
__global__ void k_relax_csr(int ncv, const int* __restrict__ nb_i, const int* __restrict__ nb_v,
                            const double* __restrict__ A, const double* __restrict__ rhs,
                            const double* __restrict__ x_in, double* __restrict__ x_out, int first) {
  int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= ncv) return;
  double acc[5];
  for (int i = 0; i < 5; i++) acc[i] = rhs[5 * c + i];
  int k0 = nb_i[c], k1 = nb_i[c + 1];
  if (!first)
    for (int k = k0 + 1; k < k1; k++) {
      int nb = nb_v[k];
      const double* Ak = A + 25 * (size_t)k;
      for (int i = 0; i < 5; i++) {
        double s = 0.0;
        for (int j = 0; j < 5; j++) s += Ak[5 * i + j] * x_in[5 * nb + j];
        acc[i] -= s;
      }
    }
  double D[25];
  for (int e = 0; e < 25; e++) D[e] = A[25 * (size_t)k0 + e];
  lu_solve5(D, acc);
  for (int i = 0; i < 5; i++) x_out[5 * c + i] = acc[i];
}

}  // namespace

extern "C" int jg_relax_csr_noalloc(int ncv, const int* nbocv_i, const int* nbocv_v, const double* A,
                                    const double* rhs, double* dq, int sweeps, void* stream) {
  if (ncv <= 0 || !nbocv_i || !nbocv_v || !A || !rhs || !dq || sweeps < 1)
    return jg::record_error(JG_ERR_ARG, "jg_relax_csr_noalloc: null pointer, ncv <= 0 or sweeps < 1");
  if (ncv > JG_NOALLOC_MAX_CELLS) {
    char msg[160];
    snprintf(msg, sizeof(msg), "jg_relax_csr_noalloc: %d cells exceed the limit of %d cells (JG_NOALLOC_MAX_CELLS)",
             ncv, JG_NOALLOC_MAX_CELLS);
    return jg::record_error(JG_ERR_ARG, msg);
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return jg::record_error(JG_ERR_NODEVICE, "jg_relax_csr_noalloc: no device");
  double* scratch = nullptr;
  if (scratch_address(dev, &scratch) != JG_OK)
    return jg::record_error(JG_ERR_CUDA, "jg_relax_csr_noalloc: cudaGetSymbolAddress of the scratch array failed");
  cudaStream_t s = (cudaStream_t)stream;
  const int tb = 128, grid = (ncv + tb - 1) / tb;
  // buffers alternate so that the last sweep writes the caller's dq
  for (int it = 0; it < sweeps; it++) {
    bool to_dq = ((sweeps - 1 - it) % 2) == 0;
    double* out = to_dq ? dq : scratch;
    const double* in = to_dq ? scratch : dq;
    k_relax_csr<<<grid, tb, 0, s>>>(ncv, nbocv_i, nbocv_v, A, rhs, in, out, it == 0);
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return jg::record_error(JG_ERR_CUDA, cudaGetErrorString(e));
  return JG_OK;
}
