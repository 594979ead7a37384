// aux_kernels.cu -- reductions, point sources and the Exner activation.
#include <cfloat>

#include "rb_common.cuh"
#include "rb_kernels.h"

namespace rb {

constexpr int RED_NT = 256;

// local_inertial.py:503-512 reduce_hmax: max(0, max h) into a zeroed slot.
__global__ void __launch_bounds__(RED_NT) max_h_kernel(const float* __restrict__ h, size_t n, unsigned int* key) {
  __shared__ float s_w[RED_NT / 32];
  float m = 0.0f;
  for (size_t k = (size_t)blockIdx.x * RED_NT + threadIdx.x; k < n; k += (size_t)gridDim.x * RED_NT) {
    const float v = h[k];
    m = v > m ? v : m;
  }
  block_max_to<RED_NT>(m, key, s_w);
}

// local_inertial.py:475-489 reduce_column_max into a zeroed slot.
__global__ void __launch_bounds__(RED_NT) max_column_kernel(const float* __restrict__ h, const float* __restrict__ w,
                                                             const float* __restrict__ d, float dx, size_t n,
                                                             unsigned int* key) {
  __shared__ float s_w[RED_NT / 32];
  float m = 0.0f;
  for (size_t k = (size_t)blockIdx.x * RED_NT + threadIdx.x; k < n; k += (size_t)gridDim.x * RED_NT) {
    const float v = column_depth(h[k], w[k], d[k], dx);
    m = v > m ? v : m;
  }
  block_max_to<RED_NT>(m, key, s_w);
}

// hllc.py:948-966 _reduce_wavespeed into a zeroed slot.
__global__ void __launch_bounds__(RED_NT) wavespeed_kernel(const float* __restrict__ h, const float* __restrict__ hu,
                                                            const float* __restrict__ hv, size_t n,
                                                            unsigned int* key) {
  __shared__ float s_w[RED_NT / 32];
  float m = 0.0f;
  for (size_t k = (size_t)blockIdx.x * RED_NT + threadIdx.x; k < n; k += (size_t)gridDim.x * RED_NT) {
    const float hh = h[k];
    const float c = sqrtf(kG * rmax(hh, 0.0f));
    const bool wet = hh > kHDry;
    const float s = wet ? rmax(div_if(wet, fabsf(hu[k]), hh), div_if(wet, fabsf(hv[k]), hh)) + c : c;
    m = s > m ? s : m;
  }
  block_max_to<RED_NT>(m, key, s_w);
}

__global__ void zero_key_kernel(unsigned int* key) { *key = 0u; }

cudaError_t reduce_max_h(const float* h, size_t n, unsigned int* key, cudaStream_t s) {
  zero_key_kernel<<<1, 1, 0, s>>>(key);
  max_h_kernel<<<WS_SUM_BLOCKS, RED_NT, 0, s>>>(h, n, key);
  return cudaGetLastError();
}

cudaError_t reduce_max_column(const float* h, const float* w, const float* d, float dx32, size_t n,
                              unsigned int* key, cudaStream_t s) {
  if (w == nullptr) return reduce_max_h(h, n, key, s);
  zero_key_kernel<<<1, 1, 0, s>>>(key);
  max_column_kernel<<<WS_SUM_BLOCKS, RED_NT, 0, s>>>(h, w, d, dx32, n, key);
  return cudaGetLastError();
}

cudaError_t reduce_wavespeed(const float* h, const float* hu, const float* hv, size_t n, unsigned int* key,
                             cudaStream_t s) {
  zero_key_kernel<<<1, 1, 0, s>>>(key);
  wavespeed_kernel<<<WS_SUM_BLOCKS, RED_NT, 0, s>>>(h, hu, hv, n, key);
  return cudaGetLastError();
}

// Deterministic float64 sum: a fixed grid of WS_SUM_BLOCKS blocks with a fixed
// element-to-thread map writes one partial each, then one block sums the
// partials in a fixed order. Same input -> same bits, every run.
template <typename T>
__global__ void __launch_bounds__(RED_NT) partial_sum_kernel(const T* __restrict__ x, size_t n, size_t stride_elems,
                                                              double* partials) {
  __shared__ double s_w[RED_NT / 32];
  double acc = 0.0;
  for (size_t k = (size_t)blockIdx.x * RED_NT + threadIdx.x; k < n; k += (size_t)gridDim.x * RED_NT)
    acc += (double)x[k * stride_elems];
  const double b = block_sum<RED_NT>(acc, s_w);
  if (threadIdx.x == 0) partials[blockIdx.x] = b;
}

__global__ void __launch_bounds__(RED_NT) final_sum_kernel(const double* partials, int np, double* out) {
  __shared__ double s_w[RED_NT / 32];
  double acc = 0.0;
  for (int k = threadIdx.x; k < np; k += RED_NT) acc += partials[k];
  const double b = block_sum<RED_NT>(acc, s_w);
  if (threadIdx.x == 0) *out = b;
}

cudaError_t sum_f64(const float* x, size_t n, double* partials, double* out, cudaStream_t s) {
  partial_sum_kernel<float><<<WS_SUM_BLOCKS, RED_NT, 0, s>>>(x, n, 1, partials);
  final_sum_kernel<<<1, RED_NT, 0, s>>>(partials, WS_SUM_BLOCKS, out);
  return cudaGetLastError();
}

// The ledger holds (total, compensation) per tile; the banked amount of a tile
// is its running total (the compensation is the rounding debt, below one ulp).
cudaError_t sum_ledger(const double* ledger, size_t nslots, double* partials, double* out, cudaStream_t s) {
  partial_sum_kernel<double><<<WS_SUM_BLOCKS, RED_NT, 0, s>>>(ledger, nslots, 2, partials);
  final_sum_kernel<<<1, RED_NT, 0, s>>>(partials, WS_SUM_BLOCKS, out);
  return cudaGetLastError();
}

// inflow.py:74-113: one thread per source entry; entries name distinct cells
// (the injector rejects duplicates), so the non-atomic add does not race.
__global__ void inject_kernel(float* h, int ny, int nx, int nsrc, const int32_t* rows, const int32_t* cols,
                              const float* add, float* comp) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= nsrc) return;
  const int r = rows[k], col = cols[k];
  if (r < 0 || r >= ny || col < 0 || col >= nx) return;  // a source outside the grid adds nothing
  const size_t c = (size_t)r * nx + col;
  if (comp != nullptr) {
    float tot = h[c], cp = comp[k];
    kahan_add(tot, cp, add[k]);
    h[c] = tot;
    comp[k] = cp;
  } else {
    h[c] = h[c] + add[k];
  }
}

// solver/processes/reservoir.py:97-121 _withdraw_pool: remove scale * h from each
// cell of the pool box and record the exact float64 depth each cell gave up.
__global__ void reservoir_withdraw_kernel(float* __restrict__ h, int nx, int r0, int c0, int rows, int cols,
                                          float scale, double* __restrict__ taken) {
  const int64_t n = (int64_t)rows * cols;
  for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x) {
    const int a = (int)(k / cols), b = (int)(k - (int64_t)a * cols);
    const size_t id = (size_t)(r0 + a) * nx + (c0 + b);
    const float avail = h[id];
    const float h_new = avail - avail * scale;
    h[id] = h_new;
    taken[k] = (double)avail - (double)h_new;
  }
}

// reservoir.py:124-144 _deliver_release: add float32(add_depth) to each outlet cell
// and bank what rounding kept from arriving (add_depth - actual gain) in the loss
// ledger. One block, fixed thread-to-cell map: the banked sum is deterministic.
__global__ void __launch_bounds__(256) reservoir_deliver_kernel(float* __restrict__ h, int nx, int r0, int c0,
                                                                int rows, int cols, double add_depth,
                                                                double* ledger_slot) {
  __shared__ double s_w[256 / 32];
  const int64_t n = (int64_t)rows * cols;
  double short_sum = 0.0;
  for (int64_t k = threadIdx.x; k < n; k += 256) {
    const int a = (int)(k / cols), b = (int)(k - (int64_t)a * cols);
    const size_t id = (size_t)(r0 + a) * nx + (c0 + b);
    const float avail = h[id];
    const float h_new = avail + (float)add_depth;
    h[id] = h_new;
    const double delivered = (double)h_new - (double)avail;
    short_sum += add_depth - delivered;
  }
  const double tot = block_sum<256>(short_sum, s_w);
  if (threadIdx.x == 0 && ledger_slot != nullptr) ledger_add(ledger_slot, tot);
}

cudaError_t reservoir_withdraw(float* h, int nx, int r0, int c0, int rows, int cols, float scale, double* taken,
                               cudaStream_t s) {
  const int64_t n = (int64_t)rows * cols;
  const int blocks = (int)((n + 255) / 256 < 1184 ? (n + 255) / 256 : 1184);
  reservoir_withdraw_kernel<<<blocks, 256, 0, s>>>(h, nx, r0, c0, rows, cols, scale, taken);
  return cudaGetLastError();
}

cudaError_t reservoir_deliver(float* h, int nx, int r0, int c0, int rows, int cols, double add_depth,
                              double* ledger_slot, cudaStream_t s) {
  reservoir_deliver_kernel<<<1, 256, 0, s>>>(h, nx, r0, c0, rows, cols, add_depth, ledger_slot);
  return cudaGetLastError();
}

cudaError_t inject_points(float* h, int ny, int nx, int nsrc, const int32_t* rows, const int32_t* cols,
                          const float* add, float* comp, cudaStream_t s) {
  if (nsrc <= 0) return cudaSuccess;
  inject_kernel<<<(nsrc + 127) / 128, 128, 0, s>>>(h, ny, nx, nsrc, rows, cols, add, comp);
  return cudaGetLastError();
}

// sediment.py:383-441 exner_update + rebuild_bed, then the integral clear of
// sediment.py:513-524 (the Kahan residues are kept).
__global__ void exner_kernel(int ny, int nx, float dx32, float inv1mp, const float* __restrict__ qs_int_x,
                             const float* __restrict__ qs_int_y, const float* __restrict__ dz_lo,
                             const float* __restrict__ dz_hi, double* dz_cum, double* dz_unapplied,
                             const float* __restrict__ z0, float* z) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  const int i = blockIdx.y;
  if (j >= nx || i >= ny) return;
  const size_t id = (size_t)i * nx + j;
  const double div_x = (double)qs_int_x[(size_t)i * (nx + 1) + j + 1] - (double)qs_int_x[(size_t)i * (nx + 1) + j];
  const double div_y = (double)qs_int_y[id + nx] - (double)qs_int_y[id];
  const double want = dz_cum[id] - (double)inv1mp * (div_x + div_y) / (double)dx32;
  double nw = want;
  const double lo = (double)dz_lo[id], hi = (double)dz_hi[id];
  if (nw < lo) nw = lo;
  if (nw > hi) nw = hi;
  if (nw != want) dz_unapplied[id] = dz_unapplied[id] + (want - nw);
  dz_cum[id] = nw;
  z[id] = (float)((double)z0[id] + nw);
}

__global__ void zero_kernel(float* a, size_t n) {
  for (size_t k = (size_t)blockIdx.x * blockDim.x + threadIdx.x; k < n; k += (size_t)gridDim.x * blockDim.x)
    a[k] = 0.0f;
}

cudaError_t exner_apply(int ny, int nx, float dx32, float inv1mp, float* qs_int_x, float* qs_int_y,
                        const float* dz_lo, const float* dz_hi, double* dz_cum, double* dz_unapplied,
                        const float* z0, float* z, cudaStream_t s) {
  const dim3 grid((nx + 127) / 128, ny);
  exner_kernel<<<grid, 128, 0, s>>>(ny, nx, dx32, inv1mp, qs_int_x, qs_int_y, dz_lo, dz_hi, dz_cum, dz_unapplied,
                                    z0, z);
  const size_t nxf = (size_t)ny * (nx + 1), nyf = (size_t)(ny + 1) * nx;
  zero_kernel<<<592, 256, 0, s>>>(qs_int_x, nxf);
  zero_kernel<<<592, 256, 0, s>>>(qs_int_y, nyf);
  return cudaGetLastError();
}

}  // namespace rb
