// Dense distance matrices of every coordinate-based TSPLIB edge type, built in HBM.
//
// Bit-identical to the reference's compute_distance_matrix / _distance_block
// (src/distances/matrix.py:44-131, 214-273) for EUC_2D/3D, MAN_2D/3D, MAX_2D/3D, CEIL_2D,
// ATT and XRAY1: every floating-point step is an explicitly rounded IEEE operation in the
// reference's order (no contraction into FMA), the sums over coordinates run left to right
// as NumPy reduces a 2- or 3-element axis, and conversions truncate like astype. GEO uses
// CUDA's double-precision cos and acos: they and the host's libm or SIMD versions may differ
// in the last bit, which changes an entry only when the value before truncation lies within
// a few ulps (about 1e-11 km) of an integer.
//
// One thread per column, its coordinates held in registers, rows strided over gridDim.y:
// each warp stores 32 consecutive int32 of a row (128-byte lines), so the kernel streams
// the n^2 * 4 output bytes at write bandwidth; the row coordinates are warp-uniform loads.
#include "common.cuh"

namespace tspb {

constexpr double kGeoPi = 3.141592;      // TSPLIB's PI (src/distances/pairwise.py:62)
constexpr double kGeoRadius = 6378.388;  // TSPLIB's earth radius in km (pairwise.py:65)

__device__ __forceinline__ double geo_radians(double x) {
  const double deg = trunc(x);
  const double minutes = __dsub_rn(x, deg);
  return __ddiv_rn(__dmul_rn(kGeoPi, __dadd_rn(deg, __ddiv_rn(__dmul_rn(5.0, minutes), 3.0))), 180.0);
}

template <int DIM>
struct Point {
  double v[DIM];
};

template <int DIM>
__device__ __forceinline__ Point<DIM> load_point(const double* __restrict__ coords, int i) {
  Point<DIM> p;
#pragma unroll
  for (int d = 0; d < DIM; ++d) p.v[d] = __ldg(coords + (long long)i * DIM + d);
  return p;
}

// Sum of squared differences over the coordinates, left to right.
template <int DIM>
__device__ __forceinline__ double sq_sum(const Point<DIM>& a, const Point<DIM>& b) {
  double s = 0.0;
#pragma unroll
  for (int d = 0; d < DIM; ++d) {
    const double t = __dsub_rn(a.v[d], b.v[d]);
    s = d == 0 ? __dmul_rn(t, t) : __dadd_rn(s, __dmul_rn(t, t));
  }
  return s;
}

template <int TYPE, int DIM>
__device__ __forceinline__ long long tsplib_distance(const Point<DIM>& a, const Point<DIM>& b) {
  if constexpr (TYPE == TSPB_EDGE_EUC_2D || TYPE == TSPB_EDGE_EUC_3D) {
    return (long long)__dadd_rn(__dsqrt_rn(sq_sum<DIM>(a, b)), 0.5);
  } else if constexpr (TYPE == TSPB_EDGE_CEIL_2D) {
    return (long long)ceil(__dsqrt_rn(sq_sum<DIM>(a, b)));
  } else if constexpr (TYPE == TSPB_EDGE_ATT) {
    const double r = __dsqrt_rn(__ddiv_rn(sq_sum<DIM>(a, b), 10.0));
    const long long t = (long long)__dadd_rn(r, 0.5);
    return (double)t < r ? t + 1 : t;
  } else if constexpr (TYPE == TSPB_EDGE_MAN_2D || TYPE == TSPB_EDGE_MAN_3D) {
    double s = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; ++d) s = d == 0 ? fabs(__dsub_rn(a.v[d], b.v[d])) : __dadd_rn(s, fabs(__dsub_rn(a.v[d], b.v[d])));
    return (long long)__dadd_rn(s, 0.5);
  } else if constexpr (TYPE == TSPB_EDGE_MAX_2D || TYPE == TSPB_EDGE_MAX_3D) {
    double m = 0.0;
#pragma unroll
    for (int d = 0; d < DIM; ++d) m = d == 0 ? fabs(__dsub_rn(a.v[d], b.v[d])) : fmax(m, fabs(__dsub_rn(a.v[d], b.v[d])));
    return (long long)__dadd_rn(m, 0.5);
  } else if constexpr (TYPE == TSPB_EDGE_GEO) {
    // a.v / b.v hold (latitude, longitude) already in radians
    const double q1 = cos(__dsub_rn(a.v[1], b.v[1]));
    const double q2 = cos(__dsub_rn(a.v[0], b.v[0]));
    const double q3 = cos(__dadd_rn(a.v[0], b.v[0]));
    double arg = __dmul_rn(0.5, __dsub_rn(__dmul_rn(__dadd_rn(1.0, q1), q2), __dmul_rn(__dsub_rn(1.0, q1), q3)));
    arg = fmin(fmax(arg, -1.0), 1.0);
    return (long long)__dadd_rn(__dmul_rn(kGeoRadius, acos(arg)), 1.0);
  } else {  // XRAY1: phi wraps at 360 degrees, motor speeds 1, scaled by 100
    const double phi = fabs(__dsub_rn(a.v[0], b.v[0]));
    const double dphi = fmin(phi, fabs(__dsub_rn(phi, 360.0)));
    const double dchi = fabs(__dsub_rn(a.v[1], b.v[1]));
    const double dth = fabs(__dsub_rn(a.v[2], b.v[2]));
    const double cost = fmax(fmax(dphi, dchi), dth);
    return (long long)(int)trunc(__dadd_rn(__dmul_rn(100.0, cost), 0.5));
  }
}

template <int TYPE, int DIM>
__global__ void __launch_bounds__(256) distance_matrix_kernel(const double* __restrict__ coords, int n,
                                                              int32_t* __restrict__ out, long long ld) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= n) return;
  Point<DIM> pc = load_point<DIM>(coords, c);
  if constexpr (TYPE == TSPB_EDGE_GEO) {
    pc.v[0] = geo_radians(pc.v[0]);
    pc.v[1] = geo_radians(pc.v[1]);
  }
  for (int r = blockIdx.y; r < n; r += gridDim.y) {
    Point<DIM> pr = load_point<DIM>(coords, r);
    if constexpr (TYPE == TSPB_EDGE_GEO) {
      pr.v[0] = geo_radians(pr.v[0]);
      pr.v[1] = geo_radians(pr.v[1]);
    }
    out[(long long)r * ld + c] = r == c ? 0 : (int32_t)tsplib_distance<TYPE, DIM>(pr, pc);
  }
}

template <int TYPE, int DIM>
static int launch_distance(const double* coords, int n, int32_t* out, long long ld, cudaStream_t st) {
  const int threads = 256;
  const dim3 grid((n + threads - 1) / threads, (unsigned)(n < 65535 ? n : 65535));
  distance_matrix_kernel<TYPE, DIM><<<grid, threads, 0, st>>>(coords, n, out, ld);
  return tspb_launch_status();
}

}  // namespace tspb

using namespace tspb;

extern "C" int tspb_distance_matrix(const double* coords, int32_t n, int32_t dim, int32_t edge_type, int32_t* out,
                                    int64_t ld, void* stream) {
  if (n < 0 || ld < n || (dim != 2 && dim != 3)) return TSPB_ERR_ARG;
  if (edge_type < TSPB_EDGE_EUC_2D || edge_type > TSPB_EDGE_XRAY1) return TSPB_ERR_ARG;
  if (edge_type == TSPB_EDGE_XRAY1 && dim != 3) return TSPB_ERR_ARG;
  if (n == 0) return TSPB_OK;
  if (!coords || !out) return TSPB_ERR_ARG;
  cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
#define TSPB_DIST_CASE(T)                                                                                   \
  case T:                                                                                                   \
    return dim == 2 ? launch_distance<T, 2>(coords, n, out, ld, st) : launch_distance<T, 3>(coords, n, out, ld, st);
  switch (edge_type) {
    TSPB_DIST_CASE(TSPB_EDGE_EUC_2D)
    TSPB_DIST_CASE(TSPB_EDGE_EUC_3D)
    TSPB_DIST_CASE(TSPB_EDGE_MAN_2D)
    TSPB_DIST_CASE(TSPB_EDGE_MAN_3D)
    TSPB_DIST_CASE(TSPB_EDGE_MAX_2D)
    TSPB_DIST_CASE(TSPB_EDGE_MAX_3D)
    TSPB_DIST_CASE(TSPB_EDGE_CEIL_2D)
    TSPB_DIST_CASE(TSPB_EDGE_ATT)
    TSPB_DIST_CASE(TSPB_EDGE_GEO)
    case TSPB_EDGE_XRAY1:
      return launch_distance<TSPB_EDGE_XRAY1, 3>(coords, n, out, ld, st);
    default:
      return TSPB_ERR_ARG;
  }
#undef TSPB_DIST_CASE
}
