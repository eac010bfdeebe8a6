// Multigrid preconditioner V-cycle (replaces _gpaw.fd_precond:
// c/fd_preconditioner.c:108-353, gpaw/preconditioner.py:59-93).
//
// The reference runs 4 stencils, 2 restrictions, 2 interpolations and 9
// elementwise passes per band (OpenMP over bands).  Here every step is one
// launch over all bands, and the elementwise passes are folded into the
// epilogues of the stencil / interpolation kernels using linearity:
//
//   reference                          this chain (8 launches)
//   r1 = R(-res)                       r1 = -R(res)
//   d1 = 4s r1; q1 = K1 d1 - r1        q1 = 4s K1 r1 - r1
//   r2 = R(q1)                         r2 = R(q1)
//   d2 = 16s r2; q2 = K2 d2 - r2;
//   d2 -= 16s q2                       d2 = 32s r2 - 256s^2 K2 r2
//   q1 = I(d2); d1 -= q1               d1 = 4s r1 - I(d2)
//   q1 = K1 d1 - r1; d1 -= 4s q1       q1 = d1 - 4s K1 d1 + 4s r1
//   d0 = I(-d1)                        q0 = -I(q1)
//   q0 = K0 d0 - res; d0 -= s q0;
//   d0 = -d0                           d0 = s K0 q0 - q0 - s res
//
// Results agree with the reference to rounding (the reassociation changes
// the last bits only).  Work arrays keep the reference's shapes; q2 and
// nresiduals are accepted for signature compatibility and not touched.
#include "internal.cuh"

using namespace gb;

static bool same3(const int64_t* a, const int64_t* b) {
  return a[0] == b[0] && a[1] == b[1] && a[2] == b[2];
}

// the V-cycle with nk phase sets (one per equal group of bands)
static int fd_precond_sets(const gb_transformer* rest0, const gb_transformer* rest1,
                           const gb_transformer* intp1, const gb_transformer* intp2,
                           const gb_operator* kin0, const gb_operator* kin1, const gb_operator* kin2,
                           void* d0, void* q0, void* r1, void* d1, void* q1, void* r2, void* d2,
                           void* q2, const void* residuals, const void* nresiduals, double step,
                           int64_t nin, int dtype, const double* phase_cd, int nk, void* stream) {
  (void)q2;
  (void)nresiduals;
  GB_REQUIRE(rest0 && rest1 && intp1 && intp2 && kin0 && kin1 && kin2,
             "gb_fd_precond: null operator/transformer");
  GB_REQUIRE(dtype_valid(dtype) && nin >= 0, "gb_fd_precond: bad dtype or batch");
  if (nin == 0) return GB_OK;
  GB_REQUIRE(d0 && q0 && r1 && d1 && q1 && r2 && d2 && residuals, "gb_fd_precond: null work array");
  GB_REQUIRE(!dtype_complex(dtype) || phase_cd, "gb_fd_precond: complex data needs phase_cd");
  GB_REQUIRE(nk >= 1 && nk <= KMAX && nin % nk == 0, "gb_fd_precond: bad number of k-point phase sets");
  GB_REQUIRE(!rest0->interpolate && !rest1->interpolate && intp1->interpolate && intp2->interpolate,
             "gb_fd_precond: transformer kinds do not match (rest0, rest1, intp1, intp2)");
  // level geometry must chain: kin0 on level 0, kin1 on level 1, kin2 on level 2
  GB_REQUIRE(same3(rest0->nin_c, kin0->n) && same3(rest0->nout_c, kin1->n) &&
                 same3(rest1->nin_c, kin1->n) && same3(rest1->nout_c, kin2->n) &&
                 same3(intp2->nin_c, kin2->n) && same3(intp2->nout_c, kin1->n) &&
                 same3(intp1->nin_c, kin1->n) && same3(intp1->nout_c, kin0->n),
             "gb_fd_precond: grid sizes of the operators do not chain");
  const bool cplx = dtype_complex(dtype);
  GB_REQUIRE(kin0->real == !cplx && kin1->real == !cplx && kin2->real == !cplx &&
                 rest0->real == !cplx && intp1->real == !cplx,
             "gb_fd_precond: real/complex flags do not match dtype");
  const double* ph = cplx ? phase_cd : nullptr;
  cudaStream_t st = (cudaStream_t)stream;
  const double s = step;
  int rc;
  Epilogue ep;

  if ((rc = tr_apply(rest0, residuals, r1, nin, dtype, ph, st, -1.0, nullptr, 0.0, nk))) return rc;
  ep = Epilogue(); ep.alpha = 4 * s; ep.beta = -1.0;
  if ((rc = op_apply(kin1, r1, q1, nin, dtype, ph, st, ep, nk))) return rc;
  if ((rc = tr_apply(rest1, q1, r2, nin, dtype, ph, st, 1.0, nullptr, 0.0, nk))) return rc;
  ep = Epilogue(); ep.alpha = -256.0 * s * s; ep.beta = 32.0 * s;
  if ((rc = op_apply(kin2, r2, d2, nin, dtype, ph, st, ep, nk))) return rc;
  if ((rc = tr_apply(intp2, d2, d1, nin, dtype, ph, st, -1.0, r1, 4 * s, nk))) return rc;
  ep = Epilogue(); ep.alpha = -4 * s; ep.beta = 1.0; ep.gamma = 4 * s; ep.y = r1;
  if ((rc = op_apply(kin1, d1, q1, nin, dtype, ph, st, ep, nk))) return rc;
  if ((rc = tr_apply(intp1, q1, q0, nin, dtype, ph, st, -1.0, nullptr, 0.0, nk))) return rc;
  ep = Epilogue(); ep.alpha = s; ep.beta = -1.0; ep.gamma = -s; ep.y = residuals;
  return op_apply(kin0, q0, d0, nin, dtype, ph, st, ep, nk);
}

extern "C" int gb_fd_precond(const gb_transformer* rest0, const gb_transformer* rest1,
                             const gb_transformer* intp1, const gb_transformer* intp2,
                             const gb_operator* kin0, const gb_operator* kin1, const gb_operator* kin2,
                             void* d0, void* q0, void* r1, void* d1, void* q1, void* r2, void* d2,
                             void* q2, const void* residuals, const void* nresiduals, double step,
                             int64_t nin, int dtype, const double* phase_cd, void* stream) {
  return fd_precond_sets(rest0, rest1, intp1, intp2, kin0, kin1, kin2, d0, q0, r1, d1, q1, r2, d2, q2,
                         residuals, nresiduals, step, nin, dtype, phase_cd, 1, stream);
}

extern "C" int gb_fd_precond_k(const gb_transformer* rest0, const gb_transformer* rest1,
                               const gb_transformer* intp1, const gb_transformer* intp2,
                               const gb_operator* kin0, const gb_operator* kin1, const gb_operator* kin2,
                               void* d0, void* q0, void* r1, void* d1, void* q1, void* r2, void* d2,
                               void* q2, const void* residuals, double step, int64_t nin, int dtype,
                               int nk, const double* phase_kcd, void* stream) {
  return fd_precond_sets(rest0, rest1, intp1, intp2, kin0, kin1, kin2, d0, q0, r1, d1, q1, r2, d2, q2,
                         residuals, nullptr, step, nin, dtype, phase_kcd, nk, stream);
}
