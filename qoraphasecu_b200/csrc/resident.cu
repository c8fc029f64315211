// Resident iteration kernel for square 2D problems of side N = 64, 128, 256.
//
// One start lives in a cluster of C CTAs (C = 1, 2, 8 for N = 64, 128, 256).
// CTA `rank` owns rows [rank R, rank R + R) of the start (R = N / C) and keeps
// in shared memory, for a whole chunk of iterations:
//   xs  the iterate's rows                 R x N complex64
//   ws  the wave rows (x-axis transform)   R x P complex64 (P padded pitch)
//   xb  the column exchange rows           R x P complex64
//   ss  the support rows                   R x N bytes
// so an iteration reads nothing from HBM but the amplitude (L2-resident, shared
// by every start). An iteration is the same sequence as the streamed passes
// (src/cuda/cuda_solver.cu:395-399 and kernels.cu:96-168 of the reference):
//   column phase: CTA `rank` owns columns [rank R, rank R + R); it gathers them
//     from every CTA's ws through distributed shared memory, transforms along
//     y, applies the modulus projection and the Fourier-error sum, transforms
//     back and scatters the columns to where they came from;
//   row phase: each CTA transforms its rows of ws back along x (= P_M x),
//     applies the update x <- S ? P : a x + b P in xs and transforms the new
//     iterate forward into ws. A row's threads share one warp and its exchange
//     reuses its own ws row, so the row transforms need warp barriers only.
// Cluster barriers separate the phases. The chunk starts from x (the forward
// row transforms are recomputed) and ends by writing x and w = FFT_x(x) to HBM,
// which keeps the invariant of the streamed passes: shrinkwrap, detwin and
// results work on the HBM copies between chunks.
//
// No thread waits on anything but hardware barriers that every thread of the
// cluster reaches the same number of times (the loop count is uniform), and
// no CTA touches another CTA's shared memory after the last cluster barrier.

#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <mutex>
#include <set>
#include <stdexcept>

#include "bulk_copy.cuh"
#include "line_fft.cuh"
#include "projection.cuh"
#include "reduce.cuh"
#include "resident.cuh"

namespace qpb {

namespace {

template <int N>
struct Resident {
  using G = Geometry<N>;
  static constexpr int C = N == 256 ? 8 : (N == 128 ? 2 : 1);
  static constexpr int E = G::E;
  static constexpr int T = G::T;
  static constexpr int R = N / C;  // rows and columns per CTA
  static constexpr int NT = R * T;
  static constexpr int P = G::PITCH;
  static constexpr int kX = R * N * 8;
  static constexpr int kW = R * P * 8;
  static constexpr int kS = R * N;
  static constexpr int kBytes = kX + 2 * kW + kS;
  static_assert(NT % 32 == 0 && NT <= 1024, "thread count");
  static_assert(kBytes + 512 <= 227 * 1024, "shared memory");
  static_assert(kS % 16 == 0, "support rows move as 16-byte vectors");
};

__device__ __forceinline__ unsigned cluster_rank() {
  unsigned r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}

// Every thread of every CTA of the cluster arrives; shared-memory writes
// before it (local and remote) are visible to every thread after it.
__device__ __forceinline__ void cluster_barrier() {
  asm volatile(
      "barrier.cluster.arrive.release.aligned;\n\t"
      "barrier.cluster.wait.acquire.aligned;" ::
          : "memory");
}

// Address in CTA `rank`'s shared memory of the same offset as `local`.
__device__ __forceinline__ unsigned cluster_map(unsigned local, unsigned rank) {
  unsigned remote;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(remote) : "r"(local), "r"(rank));
  return remote;
}

__device__ __forceinline__ float2 load_cluster(unsigned addr) {
  float2 v;
  asm volatile("ld.shared::cluster.v2.f32 {%0, %1}, [%2];" : "=f"(v.x), "=f"(v.y) : "r"(addr)
               : "memory");
  return v;
}

__device__ __forceinline__ void store_cluster(unsigned addr, float2 v) {
  asm volatile("st.shared::cluster.v2.f32 [%0], {%1, %2};" ::"r"(addr), "f"(v.x), "f"(v.y)
               : "memory");
}

template <int C>
__device__ __forceinline__ void group_barrier() {
  if constexpr (C > 1) {
    cluster_barrier();
  } else {
    __syncthreads();
  }
}

template <int N, class AmpT>
__global__ void __launch_bounds__(Resident<N>::NT, 1) resident_kernel(const ResidentParams p) {
  using K = Resident<N>;
  constexpr int C = K::C, E = K::E, T = K::T, R = K::R, P = K::P;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2* xs = reinterpret_cast<float2*>(smem_raw);
  float2* ws = xs + R * N;
  float2* xb = ws + R * P;
  auto* ss = reinterpret_cast<std::uint8_t*>(xb + R * P);

  const int tid = threadIdx.x;
  const int rank = C > 1 ? static_cast<int>(cluster_rank()) : 0;
  const int start = blockIdx.x / C;
  const long long rows_off =
      static_cast<long long>(start) * N * N + static_cast<long long>(rank) * R * N;
  const float2* __restrict__ tw = p.twiddle;
  // Row phase: T adjacent threads per row. Column phase: adjacent columns on
  // adjacent threads (a warp reads 32 neighbouring elements of one row).
  const int rl = tid / T, rt = tid % T;
  const int cl = tid % R, ct = tid / R;
  const int col = rank * R + cl;

  const Ctrl* ctrl = p.ctrl;
  const float ca = ctrl->a, cb = ctrl->b;
  const int row0 = ctrl->counters[p.group];
  const int capacity = ctrl->capacity;
  double* errs = ctrl->errs;

  {
    const auto* src = reinterpret_cast<const uint4*>(p.support + rows_off);
    auto* dst = reinterpret_cast<uint4*>(ss);
    for (int i = tid; i < K::kS / 16; i += K::NT) dst[i] = src[i];
  }
  float2 v[E];
#pragma unroll
  for (int m = 0; m < E; ++m) {
    const int j = rl * N + rt + T * m;
    v[m] = p.x[rows_off + j];
    xs[j] = v[m];
  }
  transform<N, false, true>(v, rt, tw, ws + rl * P);
#pragma unroll
  for (int m = 0; m < E; ++m) ws[rl * P + rt + T * m] = v[m];

  const unsigned ws_addr = smem_addr(ws);
  const AmpT* __restrict__ amp =
      static_cast<const AmpT*>(p.amp) +
      (p.amp_stride ? static_cast<long long>((p.start0 + start) / p.starts_per_problem) * p.amp_stride
                    : 0);
  const float scale = p.scale;
  for (int it = 0; it < p.iterations; ++it) {
    group_barrier<C>();  // every CTA's rows are transformed along x
    float a[E];
#pragma unroll
    for (int m = 0; m < E; ++m) a[m] = to_float(amp[(ct + T * m) * N + col]);
#pragma unroll
    for (int m = 0; m < E; ++m) {
      const int i = ct + T * m;
      const int owner = i / R;
      const int lr = i - owner * R;
      if constexpr (C > 1) {
        v[m] = load_cluster(cluster_map(ws_addr, owner) + static_cast<unsigned>(lr * P + col) * 8u);
      } else {
        v[m] = ws[lr * P + col];
      }
    }
    transform<N, false>(v, ct, tw, xb + cl * P);
    float acc = 0.0f;
#pragma unroll
    for (int m = 0; m < E; ++m) v[m] = pointwise_projection<Mode::kMod>(v[m], a[m], scale, acc);
    const double total = block_sum_double(static_cast<double>(acc));
    if (tid == 0) {
      const int r = row0 + it;
      if (r < capacity) {
        atomicAdd(&errs[static_cast<long long>(r) * p.starts_total + p.start0 + start], total);
      }
    }
    transform<N, true>(v, ct, tw, xb + cl * P);
#pragma unroll
    for (int m = 0; m < E; ++m) {
      const int i = ct + T * m;
      const int owner = i / R;
      const int lr = i - owner * R;
      if constexpr (C > 1) {
        store_cluster(cluster_map(ws_addr, owner) + static_cast<unsigned>(lr * P + col) * 8u, v[m]);
      } else {
        ws[lr * P + col] = v[m];
      }
    }
    group_barrier<C>();  // every column is back in its rows

#pragma unroll
    for (int m = 0; m < E; ++m) v[m] = ws[rl * P + rt + T * m];
    __syncwarp();  // a row's threads share one warp; its exchange reuses the row
    transform<N, true, true>(v, rt, tw, ws + rl * P);
#pragma unroll
    for (int m = 0; m < E; ++m) {
      const int j = rl * N + rt + T * m;
      float2 xn = v[m];
      if (!ss[j]) {
        const float2 xo = xs[j];
        xn = {ca * xo.x + cb * xn.x, ca * xo.y + cb * xn.y};
      }
      xs[j] = xn;
      v[m] = xn;
    }
    transform<N, false, true>(v, rt, tw, ws + rl * P);
#pragma unroll
    for (int m = 0; m < E; ++m) ws[rl * P + rt + T * m] = v[m];
  }

#pragma unroll
  for (int m = 0; m < E; ++m) {
    const int j = rl * N + rt + T * m;
    p.x[rows_off + j] = xs[j];
    p.w[rows_off + j] = v[m];
  }
}

__global__ void advance_counter_kernel(Ctrl* ctrl, int group, int count) {
  ctrl->counters[group] += count;
}

template <int N, class AmpT>
void launch_typed(const ResidentParams& p, int starts, cudaStream_t stream) {
  using K = Resident<N>;
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(static_cast<unsigned>(starts * K::C));
  cfg.blockDim = dim3(K::NT);
  cfg.dynamicSmemBytes = K::kBytes;
  cfg.stream = stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = K::C;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  QPB_CHECK(cudaLaunchKernelEx(&cfg, resident_kernel<N, AmpT>, p));
  count_launches(1);
}

template <int N>
void launch_side(const ResidentParams& p, int starts, cudaStream_t stream) {
  switch (p.amp_storage) {
    case AmpStorage::kF32:
      return launch_typed<N, float>(p, starts, stream);
    case AmpStorage::kF16:
      return launch_typed<N, __half>(p, starts, stream);
    case AmpStorage::kBF16:
      return launch_typed<N, __nv_bfloat16>(p, starts, stream);
  }
}

template <int N, class AmpT>
void allow_smem() {
  QPB_CHECK(cudaFuncSetAttribute(resident_kernel<N, AmpT>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 Resident<N>::kBytes));
}

template <int N>
void allow_side() {
  allow_smem<N, float>();
  allow_smem<N, __half>();
  allow_smem<N, __nv_bfloat16>();
}

template <int N>
int max_clusters_side() {
  using K = Resident<N>;
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3(static_cast<unsigned>(K::C * 64));
  cfg.blockDim = dim3(K::NT);
  cfg.dynamicSmemBytes = K::kBytes;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = K::C;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int clusters = 0;
  QPB_CHECK(cudaOccupancyMaxActiveClusters(&clusters, resident_kernel<N, float>, &cfg));
  return clusters;
}

}  // namespace

int resident_max_clusters(int side) {
  configure_resident();
  switch (side) {
    case 64: return max_clusters_side<64>();
    case 128: return max_clusters_side<128>();
    case 256: return max_clusters_side<256>();
    default: return 0;
  }
}

bool resident_supports(int ndim, int d1, int d2) {
  return ndim == 2 && d1 == d2 && (d1 == 64 || d1 == 128 || d1 == 256);
}

int resident_cluster(int side) {
  switch (side) {
    case 64: return Resident<64>::C;
    case 128: return Resident<128>::C;
    case 256: return Resident<256>::C;
    default: return 0;
  }
}

void configure_resident() {
  static std::mutex mutex;
  static std::set<int> done;
  int device = 0;
  QPB_CHECK(cudaGetDevice(&device));
  std::lock_guard<std::mutex> lock(mutex);
  if (!done.insert(device).second) return;
  allow_side<64>();
  allow_side<128>();
  allow_side<256>();
}

void launch_resident(const ResidentParams& p, int side, int starts, cudaStream_t stream) {
  if (p.iterations < 1) return;
  switch (side) {
    case 64:
      launch_side<64>(p, starts, stream);
      break;
    case 128:
      launch_side<128>(p, starts, stream);
      break;
    case 256:
      launch_side<256>(p, starts, stream);
      break;
    default:
      throw std::logic_error("resident kernel: unsupported side");
  }
  advance_counter_kernel<<<1, 1, 0, stream>>>(p.ctrl, p.group, p.iterations);
  QPB_CHECK(cudaGetLastError());
  count_launches(1);
}

}  // namespace qpb
