// Pointwise bodies of the explicit Euler residual (kernels/euler.py), for the device, templated
// on the compute type T (double under fp64, float under fp32+acc64).
//
// Every body repeats the operation order the reference's generator emits for it
// (codegen/src/autan_codegen/frontend.py, emit_cpp.py): sums of products left to right from the
// first product, min(a, b) = a <= b ? a : b, max(a, b) = a >= b ? a : b, abs(x) = x >= 0 ? x : -x,
// literals converted to T, constants folded only between two literals. The translation unit is
// compiled with --fmad=false, so no product is contracted into an FMA and each operation rounds
// once, as on the reference's host (built with -ffp-contract=off). Division and square root are the
// IEEE correctly rounded ones (nvcc's defaults). exp and log are CUDA's: their last bits may differ
// from the host C library's, so farfield and inlet states can differ in the last place.
#pragma once

#include <cuda_runtime.h>

namespace autan_b200 {

template <class T>
__device__ __forceinline__ T absv(T x) {
  return x >= T(0.0) ? x : -x;
}
template <class T>
__device__ __forceinline__ T minv(T a, T b) {
  return a <= b ? a : b;
}
template <class T>
__device__ __forceinline__ T maxv(T a, T b) {
  return a >= b ? a : b;
}
template <class T>
__device__ __forceinline__ T dot3(const T* a, const T* b) {
  return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
}

__device__ __forceinline__ float sqrt_(float x) { return sqrtf(x); }
__device__ __forceinline__ double sqrt_(double x) { return sqrt(x); }
__device__ __forceinline__ float exp_(float x) { return expf(x); }
__device__ __forceinline__ double exp_(double x) { return exp(x); }
__device__ __forceinline__ float log_(float x) { return logf(x); }
__device__ __forceinline__ double log_(double x) { return log(x); }

// Parameters of the bodies, converted to T once (they are FP64 in Data<P> and converted on use).
template <class T>
struct Params {
  T g, rgas, pref, minf;
  T ur[5];
  T scale[5];
};

// to_primitive (kernels/euler.py:94-104): W = (rho, u, v, w, p - p_ref) from dq = U - U_ref.
template <class T>
__device__ __forceinline__ void to_primitive(const T* dq, const Params<T>& p, T* w) {
  const T* ur = p.ur;
  const T rho = ur[0] + dq[0];
  const T t0 = T(2.0) * ur[1] + dq[1], t1 = T(2.0) * ur[2] + dq[2], t2 = T(2.0) * ur[3] + dq[3];
  const T dmt = dq[1] * t0 + dq[2] * t1 + dq[3] * t2;
  const T mrmr = ur[1] * ur[1] + ur[2] * ur[2] + ur[3] * ur[3];
  const T dk = (dmt * ur[0] - mrmr * dq[0]) / (rho * ur[0]);
  w[0] = rho;
  w[1] = (ur[1] + dq[1]) / rho;
  w[2] = (ur[2] + dq[2]) / rho;
  w[3] = (ur[3] + dq[3]) / rho;
  w[4] = (p.g - T(1.0)) * (dq[4] - T(0.5) * dk);
}

// total_enthalpy (:113-115).
template <class T>
__device__ __forceinline__ T enthalpy(const T* w, T g, T pr) {
  return g / (g - T(1.0)) * (w[4] + pr) / w[0] + T(0.5) * dot3(w + 1, w + 1);
}

// physical_flux (:118-130).
template <class T>
__device__ __forceinline__ void physical_flux(const T* w, const T* n, T g, T pr, T* f) {
  const T vn = dot3(w + 1, n);
  const T m = w[0] * vn;
  f[0] = m;
  f[1] = m * w[1] + w[4] * n[0];
  f[2] = m * w[2] + w[4] * n[1];
  f[3] = m * w[3] + w[4] * n[2];
  f[4] = m * enthalpy(w, g, pr);
}

// harten (:136-141).
template <class T>
__device__ __forceinline__ T harten(T lam, T delta) {
  T a = absv(lam);
  if (a < delta) a = (lam * lam + delta * delta) / (T(2.0) * delta);
  return a;
}

// roe (:144-175): Roe (1981) in the wave-strength form, Harten's fix on the acoustic waves.
template <class T>
__device__ __forceinline__ void roe(const T* wl, const T* wr, const T* n, T g, T pr, T* out) {
  const T rl = wl[0], rr = wr[0];
  const T hl = enthalpy(wl, g, pr), hr = enthalpy(wr, g, pr);
  const T s = sqrt_(rr / rl);
  const T rho = s * rl;
  const T den = T(1.0) + s;
  T v[3], dv[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    v[i] = (wl[1 + i] + s * wr[1 + i]) / den;
    dv[i] = wr[1 + i] - wl[1 + i];
  }
  const T h = (hl + s * hr) / (T(1.0) + s);
  const T vn = dot3(v, n);
  const T q2 = dot3(v, v);
  const T c = sqrt_((g - T(1.0)) * (h - T(0.5) * q2));
  const T dp = wr[4] - wl[4];
  const T drho = rr - rl;
  const T dvn = dot3(dv, n);
  const T delta = T(0.1) * c;
  const T l1 = harten(vn - c, delta);
  const T l2 = absv(vn);
  const T l5 = harten(vn + c, delta);
  const T a1 = l1 * (dp - rho * c * dvn) / (T(2.0) * c * c);
  const T a5 = l5 * (dp + rho * c * dvn) / (T(2.0) * c * c);
  const T a2 = l2 * (drho - dp / (c * c));
  const T lr = l2 * rho;
  T d[5];
  d[0] = a1 + a2 + a5;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    const T shear = dv[i] - dvn * n[i];
    d[1 + i] = a1 * (v[i] - c * n[i]) + a2 * v[i] + lr * shear + a5 * (v[i] + c * n[i]);
  }
  d[4] = a1 * (h - c * vn) + a2 * T(0.5) * q2 + lr * (dot3(v, dv) - vn * dvn) + a5 * (h + c * vn);
  T fl[5], fr[5];
  physical_flux(wl, n, g, pr, fl);
  physical_flux(wr, n, g, pr, fr);
#pragma unroll
  for (int k = 0; k < 5; ++k) out[k] = T(0.5) * (fl[k] + fr[k]) - T(0.5) * d[k];
}

// hllc_star (:178-189) minus conserved (:192-201), times the wave speed, added to the flux:
// f + sk (U*_k - U_k).
template <class T>
__device__ __forceinline__ void hllc_side(const T* w, const T* fw, const T* n, T sk, T sm, T g,
                                          T pr, T* out) {
  const T vn = dot3(w + 1, n);
  const T rs = w[0] * (sk - vn) / (sk - sm);
  const T p = w[4] + pr;
  const T vv = dot3(w + 1, w + 1);
  const T e = p / ((g - T(1.0)) * w[0]) + T(0.5) * vv;
  const T smv = sm - vn;
  T st[5], cs[5];
  st[0] = rs;
#pragma unroll
  for (int i = 0; i < 3; ++i) st[1 + i] = rs * (w[1 + i] + smv * n[i]);
  st[4] = rs * (e + (sm - vn) * (sm + p / (w[0] * (sk - vn))));
  cs[0] = w[0];
  cs[1] = w[0] * w[1];
  cs[2] = w[0] * w[2];
  cs[3] = w[0] * w[3];
  cs[4] = (w[4] + pr) / (g - T(1.0)) + T(0.5) * w[0] * vv;
#pragma unroll
  for (int k = 0; k < 5; ++k) out[k] = fw[k] + sk * (st[k] - cs[k]);
}

// hllc (:204-233): Toro, Spruce and Speares (1994) with Einfeldt's wave speeds.
template <class T>
__device__ __forceinline__ void hllc(const T* wl, const T* wr, const T* n, T g, T pr, T* out) {
  const T rl = wl[0], rr = wr[0];
  const T vnl = dot3(wl + 1, n), vnr = dot3(wr + 1, n);
  const T cl = sqrt_(g * (wl[4] + pr) / rl);
  const T cr = sqrt_(g * (wr[4] + pr) / rr);
  const T s = sqrt_(rr / rl);
  const T den = T(1.0) + s;
  T v[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) v[i] = (wl[1 + i] + s * wr[1 + i]) / den;
  const T h = (enthalpy(wl, g, pr) + s * enthalpy(wr, g, pr)) / (T(1.0) + s);
  const T c = sqrt_((g - T(1.0)) * (h - T(0.5) * dot3(v, v)));
  const T vn = dot3(v, n);
  const T sl = minv(vnl - cl, vn - c);
  const T sr = maxv(vnr + cr, vn + c);
  const T sm = (wr[4] - wl[4] + rl * vnl * (sl - vnl) - rr * vnr * (sr - vnr)) /
               (rl * (sl - vnl) - rr * (sr - vnr));
  T fl[5], fr[5];
  if (sl >= T(0.0)) {
    physical_flux(wl, n, g, pr, out);
  } else if (sm >= T(0.0)) {
    physical_flux(wl, n, g, pr, fl);
    hllc_side(wl, fl, n, sl, sm, g, pr, out);
  } else if (sr > T(0.0)) {
    physical_flux(wr, n, g, pr, fr);
    hllc_side(wr, fr, n, sr, sm, g, pr, out);
  } else {
    physical_flux(wr, n, g, pr, out);
  }
}

// Split Mach and pressure polynomials of AUSM+-up (:236-265), beta = 1/8 (16 beta folds to 2).
template <class T>
__device__ __forceinline__ T m4_plus(T m) {
  const T mp = T(0.25) * (m + T(1.0)) * (m + T(1.0));
  const T mm = T(-0.25) * (m - T(1.0)) * (m - T(1.0));
  return absv(m) >= T(1.0) ? T(0.5) * (m + absv(m)) : mp * (T(1.0) - T(2.0) * mm);
}
template <class T>
__device__ __forceinline__ T m4_minus(T m) {
  const T mp = T(0.25) * (m + T(1.0)) * (m + T(1.0));
  const T mm = T(-0.25) * (m - T(1.0)) * (m - T(1.0));
  return absv(m) >= T(1.0) ? T(0.5) * (m - absv(m)) : mm * (T(1.0) + T(2.0) * mp);
}
template <class T>
__device__ __forceinline__ T p5_plus(T m, T alpha) {
  const T mp = T(0.25) * (m + T(1.0)) * (m + T(1.0));
  const T mm = T(-0.25) * (m - T(1.0)) * (m - T(1.0));
  const T sup = m > T(0.0) ? T(1.0) : T(0.0);
  return absv(m) >= T(1.0) ? sup : mp * ((T(2.0) - m) - T(16.0) * alpha * m * mm);
}
template <class T>
__device__ __forceinline__ T p5_minus(T m, T alpha) {
  const T mp = T(0.25) * (m + T(1.0)) * (m + T(1.0));
  const T mm = T(-0.25) * (m - T(1.0)) * (m - T(1.0));
  const T sup = m < T(0.0) ? T(1.0) : T(0.0);
  return absv(m) >= T(1.0) ? sup : mm * ((T(-2.0) - m) + T(16.0) * alpha * m * mp);
}

// ausm_up (:268-303): Liou (2006), K_p = 0.25, K_u = 0.75, sigma = 1.
template <class T>
__device__ __forceinline__ void ausm(const T* wl, const T* wr, const T* n, T g, T minf, T pr,
                                     T* out) {
  const T rl = wl[0], rr = wr[0];
  const T vnl = dot3(wl + 1, n), vnr = dot3(wr + 1, n);
  const T hl = enthalpy(wl, g, pr), hr = enthalpy(wr, g, pr);
  const T csl = sqrt_(T(2.0) * (g - T(1.0)) / (g + T(1.0)) * hl);
  const T csr = sqrt_(T(2.0) * (g - T(1.0)) / (g + T(1.0)) * hr);
  const T al = csl * csl / maxv(csl, vnl);
  const T ar = csr * csr / maxv(csr, -vnr);
  const T a = minv(al, ar);
  const T ml = vnl / a;
  const T mr = vnr / a;
  const T mbar2 = T(0.5) * (vnl * vnl + vnr * vnr) / (a * a);
  const T mo2 = minv(T(1.0), maxv(mbar2, minf * minf));
  const T mo = sqrt_(mo2);
  const T fa = mo * (T(2.0) - mo);
  const T alpha = T(0.1875) * (T(-4.0) + T(5.0) * fa * fa);
  const T rho = T(0.5) * (rl + rr);
  const T mp = T(-0.25) / fa * maxv(T(1.0) - T(1.0) * mbar2, T(0.0)) * (wr[4] - wl[4]) /
               (rho * a * a);
  const T m = m4_plus(ml) + m4_minus(mr) + mp;
  const T pp = p5_plus(ml, alpha);
  const T pm = p5_minus(mr, alpha);
  const T pu = T(-0.75) * pp * pm * (rl + rr) * fa * a * (vnr - vnl);
  const T p = pp * wl[4] + pm * wr[4] + pu + (pp + pm - T(1.0)) * pr;
  const bool up = m > T(0.0);
  const T mdot = up ? a * m * rl : a * m * rr;
  const T* w = up ? wl : wr;
  const T hu = up ? hl : hr;
  out[0] = mdot;
  out[1] = mdot * w[1] + p * n[0];
  out[2] = mdot * w[2] + p * n[1];
  out[3] = mdot * w[3] + p * n[2];
  out[4] = mdot * hu;
}

// farfield_state (:309-337): Riemann invariants normal to the face.
template <class T>
__device__ __forceinline__ void farfield(const T* wi, const T* wf, const T* n, T g, T* out) {
  const T vni = dot3(wi + 1, n), vnf = dot3(wf + 1, n);
  const T ci = sqrt_(g * wi[4] / wi[0]);
  const T cf = sqrt_(g * wf[4] / wf[0]);
  if (vni >= ci) {
#pragma unroll
    for (int k = 0; k < 5; ++k) out[k] = wi[k];
    return;
  }
  if (vnf <= -cf) {
#pragma unroll
    for (int k = 0; k < 5; ++k) out[k] = wf[k];
    return;
  }
  const T rp = vni + T(2.0) * ci / (g - T(1.0));
  const T rm = vnf - T(2.0) * cf / (g - T(1.0));
  const T vnb = T(0.5) * (rp + rm);
  const T cb = T(0.25) * (g - T(1.0)) * (rp - rm);
  const bool in = vnb < T(0.0);
  const T* ws = in ? wf : wi;
  const T vns = in ? vnf : vni;
  const T ent = ws[4] / exp_(g * log_(ws[0]));
  const T rb = exp_(log_(cb * cb / (g * ent)) / (g - T(1.0)));
  out[0] = rb;
#pragma unroll
  for (int i = 0; i < 3; ++i) out[1 + i] = (ws[1 + i] - vns * n[i]) + vnb * n[i];
  out[4] = rb * cb * cb / g;
}

// inlet_state (:340-359): total pressure and temperature, flow normal to the face.
template <class T>
__device__ __forceinline__ void inlet(const T* wi, const T* data, const T* n, T g, T rgas,
                                      T* out) {
  const T p0 = data[0], t0 = data[1];
  const T gm = g - T(1.0);
  const T ci = sqrt_(g * wi[4] / wi[0]);
  const T r = dot3(wi + 1, n) + T(2.0) * ci / gm;
  const T h0 = g * rgas * t0 / gm;
  const T disc = maxv((gm + T(2.0)) * h0 - T(0.5) * gm * r * r, T(0.0));
  const T cb = gm * (r + sqrt_(disc)) / (gm + T(2.0));
  const T vnb = minv(r - T(2.0) * cb / gm, T(0.0));
  const T tb = t0 - T(0.5) * gm * vnb * vnb / (g * rgas);
  const T pb = p0 * exp_(g / gm * log_(tb / t0));
  out[0] = pb / (rgas * tb);
  out[1] = vnb * n[0];
  out[2] = vnb * n[1];
  out[3] = vnb * n[2];
  out[4] = pb;
}

// outlet_state (:362-373): static pressure, the rest from the outgoing characteristics.
template <class T>
__device__ __forceinline__ void outlet(const T* wi, const T* data, const T* n, T g, T* out) {
  const T ci = sqrt_(g * wi[4] / wi[0]);
  const T pb = data[4];
  const T dp = wi[4] - pb;
  if (dot3(wi + 1, n) >= ci) {
#pragma unroll
    for (int k = 0; k < 5; ++k) out[k] = wi[k];
    return;
  }
  const T s = dp / (wi[0] * ci);
  out[0] = wi[0] - dp / (ci * ci);
#pragma unroll
  for (int i = 0; i < 3; ++i) out[1 + i] = wi[1 + i] + s * n[i];
  out[4] = pb;
}

// boundary_value (:392-422), mirror_state (:376-380) and wall_state (:383-389) inline: a gauge
// interior state in, a gauge boundary state out; codes compared with the midpoints.
template <class T>
__device__ __forceinline__ void boundary_value(const T* wg, T kind, const T* data, const T* n,
                                               const Params<T>& p, T* out) {
  const T pr = p.pref;
  const T wi[5] = {wg[0], wg[1], wg[2], wg[3], wg[4] + pr};
  T w[5];
  T shift = pr;
  if (kind < T(0.5)) {
#pragma unroll
    for (int k = 0; k < 5; ++k) w[k] = data[k];
  } else if (kind < T(1.5)) {
    farfield(wi, data, n, p.g, w);
  } else if (kind < T(2.5)) {
    const T t = T(2.0) * dot3(wg + 1, n);
    w[0] = wg[0];
#pragma unroll
    for (int i = 0; i < 3; ++i) w[1 + i] = wg[1 + i] - t * n[i];
    w[4] = wg[4];
    shift = T(0.0) * pr;
  } else if (kind < T(3.5)) {
    inlet(wi, data, n, p.g, p.rgas, w);
  } else if (kind < T(4.5)) {
    outlet(wi, data, n, p.g, w);
  } else {
    w[0] = data[0] > T(0.0) ? (wg[4] + pr) / (p.rgas * data[0]) : wg[0];
    w[1] = T(0.0);
    w[2] = T(0.0);
    w[3] = T(0.0);
    w[4] = wg[4];
    shift = T(0.0) * pr;
  }
#pragma unroll
  for (int k = 0; k < 4; ++k) out[k] = w[k];
  out[4] = w[4] - shift;
}

// venkat (:563-567): Venkatakrishnan (1995), eq. 5.
template <class T>
__device__ __forceinline__ T venkat(T d, T dmax, T dmin, T eps2) {
  const T dp = d > T(0.0) ? dmax : dmin;
  return (dp * dp + eps2 + T(2.0) * d * dp) / (dp * dp + T(2.0) * d * d + d * dp + eps2);
}

// min(phi, venkat(d, dmax, dmin, eps2)) with the hardware min, phi <= 1, the quotient formed only
// where it can be below phi. venkat's numerator N and denominator D are >= 0 (or NaN); where
// t = fl(phi D) >= 2^-100 and N >= fl(t (1 + 2^-21)), N > phi D exactly (the two roundings lose less
// than the factor gains), so N / D > phi, its correctly rounded value is >= phi and the min is phi.
// Elsewhere (NaN, infinities, tiny products, or N / D possibly below phi) the quotient is formed as
// venkat forms it. Same bits as bound_min(phi, venkat(...)).
__device__ __forceinline__ float venkat_min(float phi, float d, float dmax, float dmin, float eps2) {
  const float dp = d > 0.0f ? dmax : dmin;
  const float num = dp * dp + eps2 + 2.0f * d * dp;
  const float den = dp * dp + 2.0f * d * d + d * dp + eps2;
  const float t = phi * den;
  if (t >= 0x1p-100f && num >= t * (1.0f + 0x1p-21f)) return phi;
  return fminf(phi, num / den);
}
__device__ __forceinline__ double venkat_min(double phi, double d, double dmax, double dmin,
                                             double eps2) {
  return fmin(phi, venkat(d, dmax, dmin, eps2));
}

// reconstruct (:619-627): W_f = W + phi (grad W . r), the cell value where rho_f or p_f + p_ref
// would not be positive.
template <class T>
__device__ __forceinline__ void reconstruct(const T* w, const T* gw, const T* lim, const T* r,
                                            T pref, T* wf) {
  T t[5];
#pragma unroll
  for (int i = 0; i < 5; ++i) {
    const T d = gw[3 * i] * r[0] + gw[3 * i + 1] * r[1] + gw[3 * i + 2] * r[2];
    t[i] = w[i] + lim[i] * d;
  }
  const bool ok = (t[0] > T(0.0)) & (t[4] + pref > T(0.0));
#pragma unroll
  for (int i = 0; i < 5; ++i) wf[i] = ok ? t[i] : w[i];
}

// flux_increment (:635-648) through axis e (its literal 0/1 components multiplied as emitted).
template <class T>
__device__ __forceinline__ void flux_increment(const T* w, const T* dw, int axis, T g, T pref,
                                               T* out) {
  const T e[3] = {axis == 0 ? T(1.0) : T(0.0), axis == 1 ? T(1.0) : T(0.0),
                  axis == 2 ? T(1.0) : T(0.0)};
  const T ve = dot3(w + 1, e);
  const T dve = dot3(dw + 1, e);
  const T vv = dot3(w + 1, w + 1);
  const T rh = g / (g - T(1.0)) * (w[4] + pref) + T(0.5) * w[0] * vv;
  const T drh = g / (g - T(1.0)) * dw[4] + T(0.5) * dw[0] * vv + w[0] * dot3(w + 1, dw + 1);
  const T dm = dw[0] * ve + w[0] * dve;
  const T wv = w[0] * ve;
  out[0] = dm;
#pragma unroll
  for (int i = 0; i < 3; ++i) out[1 + i] = dm * w[1 + i] + wv * dw[1 + i] + dw[4] * e[i];
  out[4] = drh * ve + rh * dve;
}

// warp (:651-675): the flux of the reconstruction through a warped face beyond its centroid
// value; m row-major 3 x 3.
template <class T>
__device__ __forceinline__ void warp_term(const T* w, const T* gl, const T* pl, const T* gr,
                                          const T* pr, const T* m, T g, T pref, T* out) {
  T f[3][5];
#pragma unroll
  for (int j = 0; j < 3; ++j) {
    T d[5];
#pragma unroll
    for (int i = 0; i < 5; ++i) {
      const T a = gl[3 * i] * m[j] + gl[3 * i + 1] * m[3 + j] + gl[3 * i + 2] * m[6 + j];
      const T b = gr[3 * i] * m[j] + gr[3 * i + 1] * m[3 + j] + gr[3 * i + 2] * m[6 + j];
      d[i] = T(0.5) * (pl[i] * a + pr[i] * b);
    }
    flux_increment(w, d, j, g, pref, f[j]);
  }
#pragma unroll
  for (int k = 0; k < 5; ++k) out[k] = f[0][k] + f[1][k] + f[2][k];
}

// The numerical flux chosen at compile time: 0 Roe, 1 HLLC, 2 AUSM+-up.
template <int FLUX, class T>
__device__ __forceinline__ void numerical_flux(const T* wl, const T* wr, const T* n,
                                               const Params<T>& p, T* f) {
  if constexpr (FLUX == 0) {
    roe(wl, wr, n, p.g, p.pref, f);
  } else if constexpr (FLUX == 1) {
    hllc(wl, wr, n, p.g, p.pref, f);
  } else {
    ausm(wl, wr, n, p.g, p.minf, p.pref, f);
  }
}

// The cell side's sound speed of wave_speed (:1098), the same for every face of the cell.
template <class T>
__device__ __forceinline__ T sound_speed(const T* w, T g, T pref) {
  return sqrt_(g * (w[4] + pref) / w[0]);
}

// wave_speed (:1091-1100) with the cell side's sound speed cc = sound_speed(wc) given: the same
// operations in the same order.
template <class T>
__device__ __forceinline__ T wave_speed_cc(const T* wc, T cc, const T* wn, const T* n, T area, T g,
                                           T pref) {
  const T lc = absv(dot3(wc + 1, n)) + cc;
  const T ln = absv(dot3(wn + 1, n)) + sqrt_(g * (wn[4] + pref) / wn[0]);
  return maxv(lc, ln) * area;
}

// wave_speed (:1091-1100).
template <class T>
__device__ __forceinline__ T wave_speed(const T* wc, const T* wn, const T* n, T area, T g, T pref) {
  const T lc = absv(dot3(wc + 1, n)) + sqrt_(g * (wc[4] + pref) / wc[0]);
  const T ln = absv(dot3(wn + 1, n)) + sqrt_(g * (wn[4] + pref) / wn[0]);
  return maxv(lc, ln) * area;
}

}  // namespace autan_b200
