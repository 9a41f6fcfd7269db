// The method of manufactured solutions check of the reference (mms.cc, the
// src_opt = 3 decks): a known scalar flux, the per-angle source that makes it
// the solution of the transport equation, and the comparison of the solved
// flux with it.  The O(G*C) and O(8*G*C*A) work runs on the GPU; the
// per-axis cell integrals of sin and cos (O(n) values) are computed on the
// host in the reference's order (mms.cc:35-57, 101-121, 240-275).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "internal.h"

namespace snapb200 {
namespace {

constexpr double kPi = 3.14159265358979;   // the reference's PI (snap.h:36-38)

// Cell integrals over [cb[i], cb[i+1]] of cos (cos_form = true: (cos(d cb[i]) -
// cos(d cb[i+1])) / (d del), the average of sin) or of sin ((sin(d cb[i+1]) -
// sin(d cb[i])) / del) -- mms_trigint, mms.cc:35-57.
std::vector<double> trigint(bool cos_form, int n, double d, double del, const std::vector<double> &cb) {
  std::vector<double> fn(n);
  for (int i = 0; i < n; ++i) {
    if (cos_form) {
      fn[i] = std::cos(d * cb[i]) - std::cos(d * cb[i + 1]);
      fn[i] /= d * del;
    } else {
      fn[i] = std::sin(d * cb[i + 1]) - std::sin(d * cb[i]);
      fn[i] /= del;
    }
  }
  return fn;
}

// The cell integrals along one axis of n cells split into chunks of `per`
// cells, as each chunk's task computes them (mms.cc:101-121, 240-275): the
// chunk's first edge is its first global cell index times the axis's own
// spacing `del`, the next ones step by `step` (the reference steps every axis
// by dx, which the caller passes), and the integrals use `del`.
std::vector<double> axis_trig(bool cos_form, int n, int per, double d, double del, double step) {
  std::vector<double> fn;
  fn.reserve(n);
  std::vector<double> b(per + 1);
  for (int lo = 0; lo < n; lo += per) {
    b[0] = lo * del;
    for (int i = 1; i <= per; ++i) b[i] = b[i - 1] + step;
    const std::vector<double> f = trigint(cos_form, per, d, del, b);
    fn.insert(fn.end(), f.begin(), f.end());
  }
  return fn;
}

// ref[g][c] = (g+1) tx[i] ty[j] tz[k]  (mms.cc:131-149)
__global__ void mms_flux_kernel(const double *__restrict__ tx, const double *__restrict__ ty,
                                const double *__restrict__ tz, int nx, int ny, int nz, int G,
                                double *__restrict__ ref) {
  const long long C = (long long)nx * ny * nz, n = C * G;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < n;
       idx += (long long)gridDim.x * blockDim.x) {
    const int g = (int)(idx / C);
    const long long c = idx - (long long)g * C;
    const int i = (int)(c % nx), j = (int)((c / nx) % ny), k = (int)(c / ((long long)nx * ny));
    ref[idx] = double(g + 1) * tx[i] * ty[j] * tz[k];
  }
}

// qim[o][g][c][a] (mms.cc:290-345): streaming term of the manufactured flux in
// the octant's direction, the removal sigma_t * ref, minus the scattering of
// every group into g (in-group included), in the reference's order.
__global__ void mms_source_kernel(const double *__restrict__ trig,   // cx sx | cy sy | cz sz
                                  const double *__restrict__ quad,   // mu | eta | xi [A]
                                  const double *__restrict__ ref, const int32_t *__restrict__ mat,
                                  const double *__restrict__ sigt, const double *__restrict__ slgg,
                                  int nx, int ny, int nz, int A, int G, int nmat,
                                  double *__restrict__ qim) {
  const long long C = (long long)nx * ny * nz;
  const long long n = 8LL * G * C * A;
  const double *cxv = trig, *sxv = trig + nx, *cyv = trig + 2 * nx, *syv = cyv + ny,
               *czv = cyv + 2 * ny, *szv = czv + nz;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < n;
       idx += (long long)gridDim.x * blockDim.x) {
    const int a = (int)(idx % A);
    const long long r = idx / A;
    const long long c = r % C;
    const int g = (int)((r / C) % G), o = (int)(r / (C * G));
    const double is = (o & 1) ? 1.0 : -1.0, js = (o & 2) ? 1.0 : -1.0, ks = (o & 4) ? 1.0 : -1.0;
    const int i = (int)(c % nx), j = (int)((c / nx) % ny), k = (int)(c / ((long long)nx * ny));
    const int m = mat[c] - 1;
    const double gf = double(g + 1);
    double v = 0.0;
    v += gf * is * quad[a] * sxv[i] * cyv[j] * czv[k];
    v += sigt[g * nmat + m] * ref[(size_t)g * C + c];
    v += gf * js * quad[A + a] * cxv[i] * syv[j] * czv[k];
    v += gf * ks * quad[2 * A + a] * cxv[i] * cyv[j] * szv[k];
    const double *row = slgg + ((size_t)g * nmat + m) * G;   // slgg[g][m][g'] (nmom = 1)
    for (int gp = 0; gp < G; ++gp) v -= row[gp] * ref[(size_t)gp * C + c];
    qim[idx] = v;
  }
}

// time dependent (mms.cc:387-418): qi = ref / v_g, ref *= tf - dt/2
__global__ void mms_time_kernel(double *__restrict__ ref, double *__restrict__ qi, long long C, int G,
                                double t_scale) {
  const long long n = C * G;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < n;
       idx += (long long)gridDim.x * blockDim.x) {
    const int g = (int)(idx / C);
    const double vg = double(G - g);
    const double r = ref[idx];
    qi[idx] = r / vg;
    ref[idx] = r * t_scale;
  }
}

__device__ __forceinline__ unsigned long long ordered(double x) {
  // order-preserving bits of a double (negative values flipped)
  const unsigned long long u = (unsigned long long)__double_as_longlong(x);
  return (u >> 63) ? ~u : (u | 0x8000000000000000ull);
}

// max, min, sum of |flux/ref - 1| (|flux| where ref < 1e-12), mms.cc:498-545
__global__ void mms_compare_kernel(const double *__restrict__ flux, int M,
                                   const double *__restrict__ ref, long long n,
                                   unsigned long long *__restrict__ mx,
                                   unsigned long long *__restrict__ mn, double *__restrict__ sum) {
  double lmax = -INFINITY, lmin = INFINITY, lsum = 0.0;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < n;
       idx += (long long)gridDim.x * blockDim.x) {
    const double f = flux[idx * M];
    double r = ref[idx], df = 1.0;
    if (r < 1.0e-12) {
      r = 1.0;
      df = 0.0;
    }
    df = fabs(f / r - df);
    lmax = fmax(lmax, df);
    lmin = fmin(lmin, df);
    lsum += df;
  }
  for (int off = 16; off > 0; off >>= 1) {
    lmax = fmax(lmax, __shfl_xor_sync(0xffffffffu, lmax, off));
    lmin = fmin(lmin, __shfl_xor_sync(0xffffffffu, lmin, off));
    lsum += __shfl_xor_sync(0xffffffffu, lsum, off);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMax(mx, ordered(lmax));
    atomicMin(mn, ordered(lmin));
    atomicAdd(sum, lsum);
  }
}

double from_ordered(unsigned long long u) {
  const unsigned long long b = (u >> 63) ? (u & 0x7fffffffffffffffull) : ~u;
  double x;
  std::memcpy(&x, &b, sizeof(x));
  return x;
}

int grid_of(long long n) {
  long long g = (n + 255) / 256;
  return (int)(g < 1 ? 1 : (g > 148LL * 16 ? 148LL * 16 : g));
}

}  // namespace

cudaError_t mms_init(const MmsGeometry &geo, const int32_t *mat, const double *sigt,
                     const double *slgg, double *ref, double *qim, double *qi,
                     double *scratch, cudaStream_t st) {
  const int nx = geo.nx, ny = geo.ny, nz = geo.nz;
  const double a = kPi / geo.lx, b = kPi / geo.ly, c = kPi / geo.lz;
  const double dx = geo.lx / double(nx), dy = geo.ly / double(ny), dz = geo.lz / double(nz);
  // the reference steps all three axes' edges by dx (mms.cc:104-112, 240-249)
  std::vector<double> host;
  const int *pc = geo.chunk;
  const auto cx = axis_trig(true, nx, pc[0], a, dx, dx), sx = axis_trig(false, nx, pc[0], a, dx, dx);
  const auto cy = axis_trig(true, ny, pc[1], b, dy, dx), sy = axis_trig(false, ny, pc[1], b, dy, dx);
  const auto cz = axis_trig(true, nz, pc[2], c, dz, dx), sz = axis_trig(false, nz, pc[2], c, dz, dx);
  for (const auto *v : {&cx, &sx, &cy, &sy, &cz, &sz}) host.insert(host.end(), v->begin(), v->end());
  for (int q = 0; q < 3; ++q) host.insert(host.end(), geo.quad[q], geo.quad[q] + geo.A);
  // scratch: [trig 2nx+2ny+2nz][mu eta xi 3A]
  cudaError_t e = cudaMemcpyAsync(scratch, host.data(), sizeof(double) * host.size(),
                                  cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return e;
  e = cudaStreamSynchronize(st);   // the host vector is pageable and local
  if (e != cudaSuccess) return e;
  const double *trig = scratch, *quad = scratch + 2 * (nx + ny + nz);
  const long long C = (long long)nx * ny * nz;
  // MMSInitFlux uses the cos integrals as the cell averages of sin (tx = cx)
  mms_flux_kernel<<<grid_of(C * geo.G), 256, 0, st>>>(trig, trig + 2 * nx, trig + 2 * nx + 2 * ny,
                                                     nx, ny, nz, geo.G, ref);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  mms_source_kernel<<<grid_of(8LL * geo.G * C * geo.A), 256, 0, st>>>(
      trig, quad, ref, mat, sigt, slgg, nx, ny, nz, geo.A, geo.G, geo.nmat, qim);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if (geo.timedep) {
    mms_time_kernel<<<grid_of(C * geo.G), 256, 0, st>>>(ref, qi, C, geo.G, geo.tf - 0.5 * geo.dt);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  return cudaSuccess;
}

size_t mms_scratch_words(int nx, int ny, int nz, int A) { return 2 * (size_t)(nx + ny + nz) + 3 * (size_t)A; }

cudaError_t mms_compare(const double *flux, int M, const double *ref, long long n, void *scratch,
                        double out[3], cudaStream_t st) {
  unsigned long long *mx = (unsigned long long *)scratch, *mn = mx + 1;
  double *sum = (double *)(mx + 2);
  const unsigned long long init[3] = {0ull, ~0ull, 0ull};
  cudaError_t e = cudaMemcpyAsync(scratch, init, sizeof(init), cudaMemcpyHostToDevice, st);
  if (e != cudaSuccess) return e;
  mms_compare_kernel<<<grid_of(n), 256, 0, st>>>(flux, M, ref, n, mx, mn, sum);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  unsigned long long h[3];
  e = cudaMemcpyAsync(h, scratch, sizeof(h), cudaMemcpyDeviceToHost, st);
  if (e != cudaSuccess) return e;
  if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return e;
  out[0] = from_ordered(h[0]);
  out[1] = from_ordered(h[1]);
  std::memcpy(&out[2], &h[2], sizeof(double));
  return cudaSuccess;
}

}  // namespace snapb200
