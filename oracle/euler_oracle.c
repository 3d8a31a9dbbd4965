/* CPU oracle of the explicit Euler residual-and-update path (test infrastructure only; see
 * euler_oracle.h). Built with -ffp-contract=off, as the reference's host code
 * (tests/toolchain/check_no_fma.cmake), so that every operation rounds once. */
#include "euler_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------ fp64 policy */
#define C double
#define S double
#define G double
#define GV double
#define SQRT sqrt
#define EXP exp
#define LOG log
#define SFX(name) name##_f64
#include "euler_oracle_impl.inc"
#undef C
#undef S
#undef G
#undef GV
#undef SQRT
#undef EXP
#undef LOG
#undef SFX
#undef SFX_FILL

/* ------------------------------------------------------------------ fp32+acc64 policy */
#define C float
#define S float
#define G float
#define GV float
#define SQRT sqrtf
#define EXP expf
#define LOG logf
#define SFX(name) name##_f32
#include "euler_oracle_impl.inc"
#undef C
#undef S
#undef G
#undef GV
#undef SQRT
#undef EXP
#undef LOG
#undef SFX

/* ------------------------------------------------------------------ LSQ weights */
/* Euler::Impl::compute_gradient_weights (physics/src/euler.cpp:340-416) of the owned cells: the
 * normal matrix of each cell's stencil offsets weighted by 1 / |d|^2, a boundary face in the fit
 * only with condition 0 (state) unless the fit without such faces is singular
 * (|det| <= 1e-10 |a00 a11 a22|, then every boundary face enters), an offset component within 64
 * ulps of the larger coordinate taken as zero, the inverse by cofactors over the determinant, the
 * weights s (inverse row . d). Ghost cells' weights stay 0. Here each cell's offsets are kept in a
 * scratch row between the matrix and the weights. */
typedef struct {
  double d[3];
  double s;
} lsq_offset;

static int lsq_fit(const oracle_mesh* m, int32_t c, const uint8_t* bc_kind, int every_boundary,
                   lsq_offset* row, double* w, int64_t n_stencil) {
  const int64_t first = m->stencil_offsets[c], last = m->stencil_offsets[c + 1];
  const int64_t nc = m->n_cells, nf = m->n_faces;
  double a[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int64_t k = first; k < last; ++k) {
    const int32_t e = m->stencil[k];
    const double* x;
    int64_t stride, at;
    int fit = 1;
    if (e >= 0) {
      x = m->cell_centroid;
      stride = nc;
      at = e;
    } else {
      x = m->face_centroid;
      stride = nf;
      at = -(int64_t)e - 1;
      fit = every_boundary || bc_kind[at - m->n_interior_faces] == 0;
    }
    lsq_offset* q = &row[k - first];
    for (int j = 0; j < 3; ++j) {
      const double xo = x[j * stride + at], xc = m->cell_centroid[j * nc + c];
      const double big = fabs(xo) < fabs(xc) ? fabs(xc) : fabs(xo);
      const double diff = xo - xc;
      q->d[j] = fabs(diff) <= 64 * DBL_EPSILON * big ? 0.0 : diff;
    }
    q->s = fit ? 1.0 / (q->d[0] * q->d[0] + q->d[1] * q->d[1] + q->d[2] * q->d[2]) : 0.0;
    for (int u = 0; u < 3; ++u)
      for (int v = 0; v < 3; ++v) a[3 * u + v] += q->s * q->d[u] * q->d[v];
  }
  const double det = a[0] * (a[4] * a[8] - a[5] * a[7]) - a[1] * (a[3] * a[8] - a[5] * a[6]) +
                     a[2] * (a[3] * a[7] - a[4] * a[6]);
  if (!(fabs(det) > 1e-10 * fabs(a[0] * a[4] * a[8]))) return 0;
  const double inv[9] = {(a[4] * a[8] - a[5] * a[7]) / det, (a[2] * a[7] - a[1] * a[8]) / det,
                         (a[1] * a[5] - a[2] * a[4]) / det, (a[5] * a[6] - a[3] * a[8]) / det,
                         (a[0] * a[8] - a[2] * a[6]) / det, (a[2] * a[3] - a[0] * a[5]) / det,
                         (a[3] * a[7] - a[4] * a[6]) / det, (a[1] * a[6] - a[0] * a[7]) / det,
                         (a[0] * a[4] - a[1] * a[3]) / det};
  for (int64_t k = first; k < last; ++k) {
    const lsq_offset* q = &row[k - first];
    for (int u = 0; u < 3; ++u)
      w[u * n_stencil + k] =
          q->s * (inv[3 * u] * q->d[0] + inv[3 * u + 1] * q->d[1] + inv[3 * u + 2] * q->d[2]);
  }
  return 1;
}

void oracle_gradient_weights(const oracle_mesh* m, const uint8_t* bc_kind, double* w) {
  const int64_t n_stencil = m->stencil_offsets[m->n_cells];
  memset(w, 0, (size_t)(3 * n_stencil) * sizeof(double));
  int64_t longest = 1;
  for (int32_t c = 0; c < m->n_owned_cells; ++c) {
    const int64_t len = m->stencil_offsets[c + 1] - m->stencil_offsets[c];
    if (len > longest) longest = len;
  }
  lsq_offset* row = (lsq_offset*)malloc((size_t)longest * sizeof(lsq_offset));
  for (int32_t c = 0; c < m->n_owned_cells; ++c)
    if (!lsq_fit(m, c, bc_kind, 0, row, w, n_stencil)) lsq_fit(m, c, bc_kind, 1, row, w, n_stencil);
  free(row);
}

/* ------------------------------------------------------------------ ExactSum */
/* runtime/src/exact_sum.cpp:22-140: 68 limbs of 32 bits in int64 words, limb i weighing
 * 2^(32 i - 1088); +inf, -inf and NaN counted apart; the sum rounded once, to nearest even. */
enum { LIMBS = 68, OFFSET = 1088 };
typedef struct {
  int64_t w[LIMBS + 3];
} exact_sum;

static void es_normalize(exact_sum* s) {
  for (int i = 0; i + 1 < LIMBS; ++i) {
    const int64_t carry = s->w[i] >> 32;
    s->w[i] -= carry * ((int64_t)1 << 32);
    s->w[i + 1] += carry;
  }
}

static void es_add(exact_sum* s, double t) {
  uint64_t bits;
  memcpy(&bits, &t, sizeof bits);
  const int biased = (int)((bits >> 52) & 0x7ff);
  const uint64_t fraction = bits & ((UINT64_C(1) << 52) - 1);
  const int negative = (int)(bits >> 63);
  if (biased == 0x7ff) {
    ++s->w[fraction != 0 ? LIMBS + 2 : (negative ? LIMBS + 1 : LIMBS)];
    return;
  }
  if (biased == 0 && fraction == 0) return;
  const uint64_t mant = biased == 0 ? fraction : (fraction | (UINT64_C(1) << 52));
  const int e = biased == 0 ? -1074 : biased - 1075;
  const int p = e + OFFSET;
  const int i = p >> 5, sh = p & 31;
  const uint64_t lo = (mant & 0xffffffffULL) << sh, hi = (mant >> 32) << sh;
  const int64_t sign = negative ? -1 : 1;
  s->w[i] += sign * (int64_t)(lo & 0xffffffffULL);
  s->w[i + 1] += sign * (int64_t)((lo >> 32) + (hi & 0xffffffffULL));
  s->w[i + 2] += sign * (int64_t)(hi >> 32);
}

static double es_value(const exact_sum* in) {
  if (in->w[LIMBS + 2] > 0 || (in->w[LIMBS] > 0 && in->w[LIMBS + 1] > 0)) return NAN;
  if (in->w[LIMBS] > 0) return INFINITY;
  if (in->w[LIMBS + 1] > 0) return -INFINITY;
  exact_sum a = *in;
  es_normalize(&a);
  const int negative = a.w[LIMBS - 1] < 0;
  if (negative) {
    for (int i = 0; i < LIMBS; ++i) a.w[i] = -a.w[i];
    es_normalize(&a);
  }
  int t = LIMBS - 1;
  while (t >= 0 && a.w[t] == 0) --t;
  if (t < 0) return 0.0;
#define LIMB(k) ((k) < 0 ? UINT64_C(0) : (uint64_t)a.w[(k)])
  const uint64_t top = LIMB(t);
  if (top > 0xffffffffULL) return negative ? -INFINITY : INFINITY;
  int b = 0;
  while (b < 64 && (top >> b) != 0) ++b;
  const uint64_t below = (LIMB(t - 1) << 32) | LIMB(t - 2);
  const uint64_t lead = (top << (64 - b)) | (below >> b);
  int sticky = (below & ((UINT64_C(1) << b) - 1)) != 0;
  for (int k = t - 3; k >= 0 && !sticky; --k) sticky = LIMB(k) != 0;
#undef LIMB
  uint64_t mantissa = lead >> 11;
  const uint64_t rest = lead & 0x7ff;
  if (rest > 0x400 || (rest == 0x400 && (sticky || (mantissa & 1) != 0))) ++mantissa;
  int exponent = 32 * (t - 2) - OFFSET + b + 11;
  if (mantissa == (UINT64_C(1) << 53)) {
    mantissa >>= 1;
    ++exponent;
  }
  const double magnitude = ldexp((double)mantissa, exponent);
  return negative ? -magnitude : magnitude;
}

double oracle_exact_sum(const double* terms, int64_t n) {
  exact_sum s;
  memset(&s, 0, sizeof s);
  int64_t pending = 0;
  for (int64_t i = 0; i < n; ++i) {
    es_add(&s, terms[i]);
    if (++pending == ((int64_t)1 << 29)) {
      es_normalize(&s);
      pending = 0;
    }
  }
  return es_value(&s);
}

/* record_norms (euler_physics.cpp:1040-1054): sqrt(sum R_k^2 / N) over owned cells, exact sums. */
void oracle_norms(const double* res, int32_t n_owned, int32_t n_cells, double* rms) {
  double* sq = (double*)malloc((size_t)n_owned * sizeof(double));
  const double count = (double)n_owned;
  for (int k = 0; k < 5; ++k) {
    for (int32_t c = 0; c < n_owned; ++c) {
      const double r = res[(size_t)k * (size_t)n_cells + (size_t)c];
      sq[c] = r * r;
    }
    rms[k] = sqrt(oracle_exact_sum(sq, n_owned) / count);
  }
  free(sq);
}

/* ------------------------------------------------------------------ the oracle */

struct oracle {
  oracle_mesh m;
  oracle_scheme s;
  int32_t precision;
  void* data;
  double *res, *stage, *base, *acc, *dt;
  oracle_min_fn min; /* a partitioned mesh's minimum over the ranks, or NULL */
  void* rank_user;
};

oracle* oracle_create(const oracle_mesh* mesh, const oracle_scheme* scheme, const uint8_t* bc_kind,
                      const double* bc, const double* source) {
  oracle* o = (oracle*)calloc(1, sizeof(oracle));
  o->m = *mesh;
  o->s = *scheme;
  o->precision = scheme->precision;
  if (o->precision == 0) {
    o->data = create_f64(&o->m, scheme, bc_kind, bc, source);
  } else {
    o->data = create_f32(&o->m, scheme, bc_kind, bc, source);
  }
  const size_t n5 = 5 * (size_t)mesh->n_cells;
  o->res = (double*)calloc(n5, sizeof(double));
  o->stage = (double*)calloc(n5, sizeof(double));
  o->base = (double*)calloc(n5, sizeof(double));
  o->acc = (double*)calloc(n5, sizeof(double));
  o->dt = (double*)calloc((size_t)mesh->n_cells, sizeof(double));
  return o;
}

void oracle_free(oracle* o) {
  if (o == NULL) return;
  if (o->precision == 0) {
    free_data_f64((data_f64*)o->data);
  } else {
    free_data_f32((data_f32*)o->data);
  }
  free(o->res);
  free(o->stage);
  free(o->base);
  free(o->acc);
  free(o->dt);
  free(o);
}

/* Euler<P>::set_second_order (physics/src/euler.cpp:903-912). */
void oracle_set_second_order(oracle* o, int32_t on) {
  const size_t nc = (size_t)o->m.n_cells;
  if (o->precision == 0) {
    data_f64* d = (data_f64*)o->data;
    d->second_order = on;
    if (!on) {
      memset(d->grad, 0, 15 * nc * sizeof(double));
      memset(d->phi, 0, 5 * nc * sizeof(double));
    } else if (!d->limiter) {
      for (size_t i = 0; i < 5 * nc; ++i) d->phi[i] = 1.0;
    }
  } else {
    data_f32* d = (data_f32*)o->data;
    d->second_order = on;
    if (!on) {
      memset(d->grad, 0, 15 * nc * sizeof(float));
      memset(d->phi, 0, 5 * nc * sizeof(float));
    } else if (!d->limiter) {
      for (size_t i = 0; i < 5 * nc; ++i) d->phi[i] = 1.0f;
    }
  }
}

void oracle_residual(oracle* o, const double* u, double* res) {
  if (o->precision == 0) {
    data_f64* d = (data_f64*)o->data;
    store_f64(d, u, o->s.reference);
    residual_f64(d, res, NULL);
  } else {
    data_f32* d = (data_f32*)o->data;
    store_f32(d, u, o->s.reference);
    residual_f32(d, res, NULL);
  }
}

void oracle_face_parts(oracle* o, const double* u, double* res_faces, double* face_flux) {
  const size_t n5 = 5 * (size_t)o->m.n_cells, nf5 = 5 * (size_t)o->m.n_faces;
  memset(res_faces, 0, n5 * sizeof(double));
  memset(face_flux, 0, nf5 * sizeof(double));
  if (o->precision == 0) {
    data_f64* d = (data_f64*)o->data;
    store_f64(d, u, o->s.reference);
    residual_f64(d, res_faces, face_flux);
  } else {
    data_f32* d = (data_f32*)o->data;
    store_f32(d, u, o->s.reference);
    residual_f32(d, res_faces, face_flux);
  }
}

void oracle_boundary_pressure(const oracle* o, double* p, double* force) {
  if (o->precision == 0) {
    boundary_pressure_f64((const data_f64*)o->data, p, force);
  } else {
    boundary_pressure_f32((const data_f32*)o->data, p, force);
  }
}

#define COPY_OUT(dst, src, n)                                          \
  do {                                                                 \
    if ((dst) != NULL)                                                 \
      for (size_t i_ = 0; i_ < (n); ++i_) (dst)[i_] = (double)(src)[i_]; \
  } while (0)

void oracle_arrays(const oracle* o, double* prim, double* grad, double* phi, double* wmin,
                   double* wmax, double* prim_b) {
  const size_t nc = (size_t)o->m.n_cells, nf = (size_t)o->m.n_faces;
  if (o->precision == 0) {
    const data_f64* d = (const data_f64*)o->data;
    COPY_OUT(prim, d->prim, 5 * nc);
    COPY_OUT(grad, d->grad, 15 * nc);
    COPY_OUT(phi, d->phi, 5 * nc);
    COPY_OUT(wmin, d->wmin, 5 * nc);
    COPY_OUT(wmax, d->wmax, 5 * nc);
    COPY_OUT(prim_b, d->prim_b, 5 * nf);
  } else {
    const data_f32* d = (const data_f32*)o->data;
    COPY_OUT(prim, d->prim, 5 * nc);
    COPY_OUT(grad, d->grad, 15 * nc);
    COPY_OUT(phi, d->phi, 5 * nc);
    COPY_OUT(wmin, d->wmin, 5 * nc);
    COPY_OUT(wmax, d->wmax, 5 * nc);
    COPY_OUT(prim_b, d->prim_b, 5 * nf);
  }
}

/* The values of a rank's external ghosts for the next residual (see the data's ext_* fields):
 * 5, 15 and 5 x ghosts, ghost order, entries of periodic images unused; the arrays stay the
 * caller's and must outlive the evaluations that read them. */
void oracle_set_external(oracle* o, const double* prim, const double* grad, const double* phi) {
  if (o->precision == 0) {
    data_f64* d = (data_f64*)o->data;
    d->ext_prim = prim, d->ext_grad = grad, d->ext_phi = phi;
  } else {
    data_f32* d = (data_f32*)o->data;
    d->ext_prim = prim, d->ext_grad = grad, d->ext_phi = phi;
  }
}

void oracle_set_ranks(oracle* o, oracle_halo_fn halo, oracle_min_fn min, void* user) {
  o->min = min;
  o->rank_user = user;
  if (o->precision == 0) {
    data_f64* d = (data_f64*)o->data;
    d->halo = halo, d->halo_user = user;
  } else {
    data_f32* d = (data_f32*)o->data;
    d->halo = halo, d->halo_user = user;
  }
}

void oracle_spectral_radius(oracle* o, double* lambda) {
  const size_t nc = (size_t)o->m.n_cells;
  if (o->precision == 0) {
    data_f64* d = (data_f64*)o->data;
    spectral_f64(d);
    COPY_OUT(lambda, d->lam, nc);
  } else {
    data_f32* d = (data_f32*)o->data;
    spectral_f32(d);
    COPY_OUT(lambda, d->lam, nc);
  }
}

int64_t oracle_first_invalid(const oracle* o, const double* u, const double* res) {
  const size_t nc = (size_t)o->m.n_cells;
  for (int32_t c = 0; c < o->m.n_owned_cells; ++c) {
    const int bad = o->precision == 0
                        ? invalid_state_f64(u, nc, (size_t)c, o->s.reference, o->s.gamma)
                        : invalid_state_f32(u, nc, (size_t)c, o->s.reference, o->s.gamma);
    if (bad) return c;
  }
  for (int32_t c = 0; c < o->m.n_owned_cells; ++c)
    for (int k = 0; k < 5; ++k)
      if (!isfinite(res[(size_t)k * nc + (size_t)c])) return c;
  return -1;
}

/* One explicit step.
 * rk == 3: SSP-RK3 of Shu and Osher (1988) eq. 2.18 as EulerPhysics::unsteady_step
 *   (euler_physics.cpp:1362-1393) and CudaStepper::step (device_stepper.cuh:313-345):
 *   next = stage - (h / V) R(stage); stage = a u + b next, (a, b) = (0, 1), (3/4, 1/4), (1/3, 2/3).
 * rk == 4: classical RK4 (Kutta 1901), not in the reference, in the same operation style:
 *   stage_s = u - ((c_s dt) / V) R_{s-1} with c = (1/2, 1/2, 1); acc = R_0, acc = acc + 2 R_1,
 *   acc = acc + 2 R_2, acc = acc + R_3; u = u - ((dt / 6) / V) acc.
 * The global step is min over owned cells of (CFL V) / lambda (euler_physics.cpp:1370-1377); with
 * `local`, each cell takes its own (CFL V) / lambda. */
int64_t oracle_step(oracle* o, double* u, int32_t rk, double cfl, double dt, int32_t local,
                    double* norms, double* dt_out) {
  const size_t nc = (size_t)o->m.n_cells;
  const int32_t owned = o->m.n_owned_cells;
  const double* vol = o->m.cell_volume;
  double* res = o->res;
  oracle_residual(o, u, res);
  if (norms != NULL) oracle_norms(res, owned, o->m.n_cells, norms);
  double h = dt;
  if (!(dt > 0.0)) {
    double* lam = o->dt;
    oracle_spectral_radius(o, lam);
    h = INFINITY;
    for (int32_t c = 0; c < owned; ++c) {
      const double t = cfl * vol[c] / lam[c];
      lam[c] = t;
      h = fmin(h, t);
    }
    if (o->min != NULL) o->min(o->rank_user, &h);  /* Ranks::min of the step */
  }
  if (dt_out != NULL) *dt_out = h;
  const int use_local = !(dt > 0.0) && local;
  memcpy(o->stage, u, 5 * nc * sizeof(double));
  if (rk == 3) {
    static const double w[3][2] = {{0.0, 1.0}, {0.75, 0.25}, {1.0 / 3.0, 2.0 / 3.0}};
    for (int s = 0; s < 3; ++s) {
      if (s > 0) oracle_residual(o, o->stage, res);
      for (int k = 0; k < 5; ++k)
        for (int32_t c = 0; c < owned; ++c) {
          const size_t i = (size_t)k * nc + (size_t)c;
          const double hc = use_local ? o->dt[c] : h;
          const double next = o->stage[i] - hc / vol[c] * res[i];
          o->stage[i] = w[s][0] * u[i] + w[s][1] * next;
        }
    }
    for (int k = 0; k < 5; ++k)
      for (int32_t c = 0; c < owned; ++c) u[(size_t)k * nc + c] = o->stage[(size_t)k * nc + c];
  } else {
    static const double cs[3] = {0.5, 0.5, 1.0};
    for (int s = 0; s < 4; ++s) {
      if (s > 0) oracle_residual(o, o->stage, res);
      for (int k = 0; k < 5; ++k)
        for (int32_t c = 0; c < owned; ++c) {
          const size_t i = (size_t)k * nc + (size_t)c;
          const double hc = use_local ? o->dt[c] : h;
          if (s == 0) {
            o->acc[i] = res[i];
          } else if (s < 3) {
            o->acc[i] = o->acc[i] + 2.0 * res[i];
          } else {
            o->acc[i] = o->acc[i] + res[i];
          }
          if (s < 3) {
            o->stage[i] = u[i] - cs[s] * hc / vol[c] * res[i];
          } else {
            o->stage[i] = u[i] - hc / 6.0 / vol[c] * o->acc[i];
          }
        }
    }
    for (int k = 0; k < 5; ++k)
      for (int32_t c = 0; c < owned; ++c) u[(size_t)k * nc + c] = o->stage[(size_t)k * nc + c];
  }
  /* CudaStepper::invalid (device_stepper.cuh:468-491): the new state, then the residual of the
   * last stage. */
  return oracle_first_invalid(o, u, res);
}

/* ------------------------------------------------------------------ pointwise bodies */

static void params_f64(const oracle_scheme* s, par_f64* p) {
  const double* r = s->reference;
  p->g = s->gamma;
  p->rgas = s->gas_constant;
  p->minf = s->mach_ref;
  p->pref = (s->gamma - 1.0) * (r[4] - 0.5 * (r[1] * r[1] + r[2] * r[2] + r[3] * r[3]) / r[0]);
  for (int c = 0; c < 5; ++c) p->ur[c] = r[c];
}

static void params_f32(const oracle_scheme* s, par_f32* p) {
  const double* r = s->reference;
  p->g = (float)s->gamma;
  p->rgas = (float)s->gas_constant;
  p->minf = (float)s->mach_ref;
  p->pref = (float)((s->gamma - 1.0) * (r[4] - 0.5 * (r[1] * r[1] + r[2] * r[2] + r[3] * r[3]) / r[0]));
  for (int c = 0; c < 5; ++c) p->ur[c] = (float)r[c];
}

void oracle_flux(const oracle_scheme* s, const double* wl, const double* wr, const double* n,
                 double* out) {
  if (s->precision == 0) {
    par_f64 p;
    params_f64(s, &p);
    double f[5];
    if (s->flux == 0) roe_f64(wl, wr, n, p.g, p.pref, f);
    else if (s->flux == 1) hllc_f64(wl, wr, n, p.g, p.pref, f);
    else ausm_f64(wl, wr, n, p.g, p.minf, p.pref, f);
    for (int k = 0; k < 5; ++k) out[k] = f[k];
  } else {
    par_f32 p;
    params_f32(s, &p);
    float a[5], b[5], nn[3], f[5];
    for (int k = 0; k < 5; ++k) {
      a[k] = (float)wl[k];
      b[k] = (float)wr[k];
    }
    for (int k = 0; k < 3; ++k) nn[k] = (float)n[k];
    if (s->flux == 0) roe_f32(a, b, nn, p.g, p.pref, f);
    else if (s->flux == 1) hllc_f32(a, b, nn, p.g, p.pref, f);
    else ausm_f32(a, b, nn, p.g, p.minf, p.pref, f);
    for (int k = 0; k < 5; ++k) out[k] = f[k];
  }
}

void oracle_boundary_value(const oracle_scheme* s, const double* wg, double kind,
                           const double* data, const double* n, double* out) {
  if (s->precision == 0) {
    par_f64 p;
    params_f64(s, &p);
    boundary_value_f64(wg, kind, data, n, p.g, p.rgas, p.pref, out);
  } else {
    par_f32 p;
    params_f32(s, &p);
    float a[5], d[5], nn[3], f[5];
    for (int k = 0; k < 5; ++k) {
      a[k] = (float)wg[k];
      d[k] = (float)data[k];
    }
    for (int k = 0; k < 3; ++k) nn[k] = (float)n[k];
    boundary_value_f32(a, (float)kind, d, nn, p.g, p.rgas, p.pref, f);
    for (int k = 0; k < 5; ++k) out[k] = f[k];
  }
}

void oracle_to_primitive(const oracle_scheme* s, const double* dq, double* out) {
  if (s->precision == 0) {
    par_f64 p;
    params_f64(s, &p);
    to_primitive_f64(dq, p.ur, p.g, out);
  } else {
    par_f32 p;
    params_f32(s, &p);
    float a[5], f[5];
    for (int k = 0; k < 5; ++k) a[k] = (float)(float)dq[k];
    to_primitive_f32(a, p.ur, p.g, f);
    for (int k = 0; k < 5; ++k) out[k] = f[k];
  }
}
