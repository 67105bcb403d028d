// ref_shim.cu -- TEST INFRASTRUCTURE ONLY.
//
// Compiles the reference engine (src/cuda/leviathan_kernel.cu of the
// reference, unmodified, pulled in with #include from its own location by
// oracle/Makefile) into oracle/_ref/, and adds read-only accessors for the
// state the reference ABI does not expose (weights, predictor, ring, buffer
// index; leviathan_kernel.cu:27-72).  Used by tests/ and by the reference arm
// of bench.py to run the reference engine on the same GPU and the same
// inputs as this repository's engine.
#include "leviathan_kernel.cu"

extern "C" {

// Copies the reference engine's device state to host buffers (any may be
// null).  ring is node-major [N][max_delay+1] as in the reference.
int ref_shim_get_state(LeviathanHandle *h, float *theta, float *theta_hat,
                       float *omega_hat, float *weights, float *ring,
                       int *buf_idx, float *g) {
  if (!h) return -1;
  cudaStreamSynchronize(h->stream);
  cudaError_t e = cudaSuccess;
  if (theta && e == cudaSuccess)
    e = cudaMemcpy(theta, h->d_theta, sizeof(float) * h->N,
                   cudaMemcpyDeviceToHost);
  if (theta_hat && e == cudaSuccess)
    e = cudaMemcpy(theta_hat, h->d_theta_hat, sizeof(float) * h->N,
                   cudaMemcpyDeviceToHost);
  if (omega_hat && e == cudaSuccess)
    e = cudaMemcpy(omega_hat, h->d_omega_hat, sizeof(float) * h->N,
                   cudaMemcpyDeviceToHost);
  if (weights && e == cudaSuccess && h->num_edges > 0)
    e = cudaMemcpy(weights, h->d_weights, sizeof(float) * h->num_edges,
                   cudaMemcpyDeviceToHost);
  if (ring && e == cudaSuccess)
    e = cudaMemcpy(ring, h->d_theta_buffer,
                   sizeof(float) * (size_t)h->N * h->buffer_size,
                   cudaMemcpyDeviceToHost);
  if (buf_idx) *buf_idx = h->buf_idx;
  if (g) *g = h->g;
  return e == cudaSuccess ? 0 : -2;
}

// Stream of the reference engine (for timing with CUDA events).
void *ref_shim_stream(LeviathanHandle *h) {
  return h ? reinterpret_cast<void *>(h->stream) : nullptr;
}

}  // extern "C"
