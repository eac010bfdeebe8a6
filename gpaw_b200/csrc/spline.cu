// Radial splines and spline_to_grid on the device (replaces _gpaw.Spline,
// c/spline.c, and _gpaw.spline_to_grid, c/lfc.c:887-977).
//
// gb_spline_new builds the natural cubic spline of c/bmgs/spline.c:11-47
// (zero slope at r = 0, the same tridiagonal recurrences, coefficients per
// bin) on the host and keeps the coefficient table in device memory.
//
// gb_spline_to_grid tabulates f(r) r^l Y_lm on a box of grid points around
// a centre and lists the grid runs it covers, as the reference does: rows
// (g0, g1) in order, along each row the points with r < rmax (a contiguous
// run, the intersection of a line with a ball), A_gm rows in that order and
// G_B = [start, end) pairs of the runs in the flat index of the local grid.
// Three launches on the caller's stream:
//   spline_rows_kernel   one thread per row finds the row's run
//   spline_scan_kernel   one CTA prefix-sums the run lengths and counts runs
//   spline_fill_kernel   one CTA per row writes its run's values and bounds
// The run bounds are found by the same distance test as the reference
// (see spline.cuh on rounding), so the runs are identical, not just close.
#include <vector>

#include "internal.cuh"
#include "spline.cuh"

namespace gb {

SplineDev spline_view(const gb_spline* s) { return SplineDev{s->coef, s->nbins, s->l, s->dr}; }

namespace {

struct BoxArgs {
  SplineDev s;
  int64_t beg[3], end[3];
  double pos[3];
  double h[9];
  int64_t n[3], corner[3];
  double rcut;
  int nm;
};

// grid point (g0, g1, g2) relative to the centre, and its distance
__device__ __forceinline__ void rel_point(const BoxArgs& a, int64_t g0, int64_t g1, int64_t g2, double& x,
                                          double& y, double& z, double& r2) {
  const double d0 = (double)g0, d1 = (double)g1, d2 = (double)g2;
  x = sub_(add_(add_(mul_(a.h[0], d0), mul_(a.h[3], d1)), mul_(a.h[6], d2)), a.pos[0]);
  y = sub_(add_(add_(mul_(a.h[1], d0), mul_(a.h[4], d1)), mul_(a.h[7], d2)), a.pos[1]);
  z = sub_(add_(add_(mul_(a.h[2], d0), mul_(a.h[5], d1)), mul_(a.h[8], d2)), a.pos[2]);
  r2 = add_(add_(mul_(x, x), mul_(y, y)), mul_(z, z));
}

__global__ void spline_rows_kernel(const BoxArgs a, int64_t nrows, int n1b, int* first, int* len) {
  const int64_t row = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (row >= nrows) return;
  const int64_t g0 = a.beg[0] + row / n1b, g1 = a.beg[1] + row % n1b;
  int lo = -1, hi = -1;
  for (int64_t g2 = a.beg[2]; g2 < a.end[2]; ++g2) {
    double x, y, z, r2;
    rel_point(a, g0, g1, g2, x, y, z, r2);
    if (__dsqrt_rn(r2) < a.rcut) {
      if (lo < 0) lo = (int)g2;
      hi = (int)g2;
    }
  }
  first[row] = lo;
  len[row] = lo < 0 ? 0 : hi - lo + 1;
}

// exclusive prefix sums of the run lengths (offset in rows of A) and of
// the non-empty rows (run index), totals into counts = {points, 2 * runs}
__global__ void __launch_bounds__(1024) spline_scan_kernel(const int* len, int64_t nrows, int64_t* off,
                                                            int* run, int64_t* counts) {
  __shared__ int64_t s_pts[1024];
  __shared__ int s_runs[1024];
  const int t = threadIdx.x;
  const int64_t chunk = (nrows + 1023) / 1024;
  const int64_t r0 = t * chunk, r1 = r0 + chunk < nrows ? r0 + chunk : nrows;
  int64_t p = 0;
  int q = 0;
  for (int64_t r = r0; r < r1; ++r) {
    p += len[r];
    q += len[r] > 0;
  }
  s_pts[t] = p;
  s_runs[t] = q;
  __syncthreads();
  if (t == 0) {
    int64_t ap = 0;
    int aq = 0;
    for (int i = 0; i < 1024; ++i) {
      const int64_t vp = s_pts[i];
      const int vq = s_runs[i];
      s_pts[i] = ap;
      s_runs[i] = aq;
      ap += vp;
      aq += vq;
    }
    counts[0] = ap;
    counts[1] = 2 * (int64_t)aq;
  }
  __syncthreads();
  p = s_pts[t];
  q = s_runs[t];
  for (int64_t r = r0; r < r1; ++r) {
    off[r] = p;
    run[r] = q;
    p += len[r];
    q += len[r] > 0;
  }
}

__global__ void spline_fill_kernel(const BoxArgs a, int n1b, const int* first, const int* len,
                                   const int64_t* off, const int* run, double* A, int* G_B) {
  const int64_t row = blockIdx.x;
  const int nl = len[row];
  if (nl == 0) return;
  const int64_t g0 = a.beg[0] + row / n1b, g1 = a.beg[1] + row % n1b;
  const int lo = first[row];
  if (threadIdx.x == 0) {
    const int64_t G = ((g0 - a.corner[0]) * a.n[1] + (g1 - a.corner[1])) * a.n[2] - a.corner[2];
    G_B[2 * run[row]] = (int)(G + lo);
    G_B[2 * run[row] + 1] = (int)(G + lo + nl);
  }
  for (int k = threadIdx.x; k < nl; k += blockDim.x) {
    double x, y, z, r2;
    rel_point(a, g0, g1, lo + k, x, y, z, r2);
    const double f = spline_value(a.s, __dsqrt_rn(r2));
    double p[5];
    solid_harmonics(a.s.l, f, x, y, z, r2, p);
    double* out = A + (off[row] + k) * a.nm;
    for (int m = 0; m < a.nm; ++m) out[m] = p[m];
  }
}

}  // namespace
}  // namespace gb

using namespace gb;

extern "C" {

int gb_spline_new(int l, double rmax, int nbins, const double* f_g, gb_spline** out) {
  GB_REQUIRE(out && f_g, "gb_spline_new: null argument");
  GB_REQUIRE(l >= 0 && l <= 2, "gb_spline_new: l must be 0, 1 or 2");
  GB_REQUIRE(nbins >= 1 && rmax > 0.0, "gb_spline_new: needs nbins >= 1 and rmax > 0");
  // natural cubic spline through f at r = b dr with zero slope at r = 0
  // (the recurrences of c/bmgs/spline.c:11-47)
  const double dr = rmax / nbins;
  const double c = 3.0 / (dr * dr);
  std::vector<double> f2(nbins + 1), u(nbins), s(4 * (size_t)(nbins + 1), 0.0);
  f2[0] = -0.5;
  u[0] = (f_g[1] - f_g[0]) * c;
  for (int b = 1; b < nbins; ++b) {
    const double p = 0.5 * f2[b - 1] + 2.0;
    f2[b] = -0.5 / p;
    u[b] = ((f_g[b + 1] - 2.0 * f_g[b] + f_g[b - 1]) * c - 0.5 * u[b - 1]) / p;
  }
  f2[nbins] = (f_g[nbins - 1] * c - 0.5 * u[nbins - 1]) / (0.5 * f2[nbins - 1] + 1.0);
  for (int b = nbins - 1; b >= 0; --b) f2[b] = f2[b] * f2[b + 1] + u[b];
  for (int b = 0; b < nbins; ++b) {
    s[4 * b + 0] = f_g[b];
    s[4 * b + 1] = (f_g[b + 1] - f_g[b]) / dr - (f2[b] / 3 + f2[b + 1] / 6) * dr;
    s[4 * b + 2] = 0.5 * f2[b];
    s[4 * b + 3] = (f2[b + 1] - f2[b]) / (6 * dr);
  }
  gb_spline* sp = new gb_spline;
  sp->l = l;
  sp->nbins = nbins;
  sp->rmax = rmax;
  sp->dr = dr;
  if (cudaMalloc(&sp->coef, s.size() * sizeof(double)) != cudaSuccess) {
    delete sp;
    return fail(GB_E_NOMEM, "gb_spline_new: cudaMalloc failed");
  }
  if (cudaMemcpy(sp->coef, s.data(), s.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) {
    cudaFree(sp->coef);
    delete sp;
    return fail(GB_E_CUDA, "gb_spline_new: upload failed");
  }
  *out = sp;
  return GB_OK;
}

int gb_spline_free(gb_spline* s) {
  if (!s) return GB_OK;
  cudaFree(s->coef);
  delete s;
  return GB_OK;
}

int gb_spline_get(const gb_spline* s, int* l, double* rmax, int* nbins) {
  GB_REQUIRE(s, "gb_spline_get: null spline");
  if (l) *l = s->l;
  if (rmax) *rmax = s->rmax;
  if (nbins) *nbins = s->nbins;
  return GB_OK;
}

int gb_spline_to_grid(const gb_spline* s, const int64_t beg_c[3], const int64_t end_c[3],
                      const double pos_v[3], const double h_cv[9], const int64_t n_c[3],
                      const int64_t gdcorner_c[3], double* A_gm, int* G_B, int64_t* ng_out,
                      int64_t* nB_out, void* stream) {
  GB_REQUIRE(s && beg_c && end_c && pos_v && h_cv && n_c && gdcorner_c && ng_out && nB_out,
             "gb_spline_to_grid: null argument");
  BoxArgs a;
  int64_t ext[3];
  for (int c = 0; c < 3; ++c) {
    a.beg[c] = beg_c[c];
    a.end[c] = end_c[c];
    a.pos[c] = pos_v[c];
    a.n[c] = n_c[c];
    a.corner[c] = gdcorner_c[c];
    ext[c] = end_c[c] - beg_c[c];
    GB_REQUIRE(n_c[c] > 0 && beg_c[c] >= gdcorner_c[c] && end_c[c] <= gdcorner_c[c] + n_c[c],
               "gb_spline_to_grid: box outside the local grid");
  }
  for (int i = 0; i < 9; ++i) a.h[i] = h_cv[i];
  a.s = spline_view(s);
  a.rcut = s->dr * s->nbins;
  a.nm = 2 * s->l + 1;
  *ng_out = 0;
  *nB_out = 0;
  if (ext[0] <= 0 || ext[1] <= 0 || ext[2] <= 0) return GB_OK;
  GB_REQUIRE(A_gm && G_B, "gb_spline_to_grid: null output");
  GB_REQUIRE(n_c[0] * n_c[1] * n_c[2] < ((int64_t)1 << 31) && ext[1] < (1 << 30),
             "gb_spline_to_grid: grid too large for int32 indices");
  const int64_t nrows = ext[0] * ext[1];
  cudaStream_t st = (cudaStream_t)stream;
  // work arrays: first, len, run (int) and off (int64) per row, counts
  void* work = nullptr;
  const size_t wbytes = (size_t)nrows * (3 * sizeof(int) + sizeof(int64_t)) + 2 * sizeof(int64_t) + 64;
  if (cudaMallocAsync(&work, wbytes, st) != cudaSuccess)
    return fail(GB_E_NOMEM, "gb_spline_to_grid: work space allocation failed");
  int64_t* off = static_cast<int64_t*>(work);
  int64_t* counts = off + nrows;
  int* first = reinterpret_cast<int*>(counts + 2);
  int* len = first + nrows;
  int* run = len + nrows;
  const int n1b = (int)ext[1];
  spline_rows_kernel<<<(unsigned)((nrows + 127) / 128), 128, 0, st>>>(a, nrows, n1b, first, len);
  int rc = check_launch("spline_rows_kernel");
  if (!rc) {
    spline_scan_kernel<<<1, 1024, 0, st>>>(len, nrows, off, run, counts);
    rc = check_launch("spline_scan_kernel");
  }
  if (!rc) {
    spline_fill_kernel<<<(unsigned)nrows, 64, 0, st>>>(a, n1b, first, len, off, run, A_gm, G_B);
    rc = check_launch("spline_fill_kernel");
  }
  int64_t h_counts[2] = {0, 0};
  if (!rc && cudaMemcpyAsync(h_counts, counts, sizeof(h_counts), cudaMemcpyDeviceToHost, st) != cudaSuccess)
    rc = fail(GB_E_CUDA, "gb_spline_to_grid: count read-back failed");
  cudaFreeAsync(work, st);
  if (!rc && cudaStreamSynchronize(st) != cudaSuccess) rc = fail(GB_E_CUDA, "gb_spline_to_grid: sync failed");
  if (rc) return rc;
  *ng_out = h_counts[0];
  *nB_out = h_counts[1];
  return GB_OK;
}

}  // extern "C"
