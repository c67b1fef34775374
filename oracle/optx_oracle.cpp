// optx_oracle.cpp - CPU restatement of the reference optical-photon transport.
//
// TEST INFRASTRUCTURE ONLY. This file is the checker for the CUDA engine in
// gpu_optical_photons_b200/csrc: only tests/, __graft_entry__.smoke() and
// bench.py's cpu_baseline leg load it. No product code path links or calls it.
//
// It restates, step by step, the physics of the reference project
// zmeskma/GPU_Optical_photons (paths relative to that project):
//   include/optphot/philox.hpp     Philox4x32-10, u32_to_uniform, PhiloxStream
//   include/optphot/pmath.hpp      platform / portable log, sincos(turns), cbrt
//   include/optphot/vec3.hpp       Vec3, orthonormal_basis, rotate_about
//   include/optphot/geometry.hpp   distance_to_box_exit, face_normal, snap_to_face
//   include/optphot/fresnel.hpp    fresnel_unpolarized, reflect
//   include/optphot/sampling.hpp   exponential, isotropic, Rayleigh, Lambertian
//   include/optphot/transport.hpp  start_photon, step_photon, transport_photon,
//                                  time_bin, xy_bin
//   src/cpu/cpu_backend.cpp        records / tally loops
// with the same floating-point expression order, so that, compiled with
// -ffp-contract=off, it reproduces the reference CPU build bit for bit (pinned
// by tests/test_oracle_golden.py against the reference compiled from its own
// sources, and by the golden fixtures in tests/golden/).
//
// Extensions beyond the reference (each keeps the reference draw order):
//   * per-face surfaces (faces 0..4 each with their own model / reflectivity);
//   * batched events (per-event parameters, global photon id = offset + local);
//   * score-function terms for the adjoint gradient (FP64);
//   * a double-precision transport (Real = double) and an op-counting scalar
//     type (Real = Counted) used to pin the algorithmic work per photon-step.
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <vector>

#if defined(_OPENMP)
#include <omp.h>
#endif

namespace oracle {

// ---------------------------------------------------------------------------
// Parameters: byte layout of SimParams (include/optphot/params.hpp:40-63).
struct Params {
  float hx, hy, hz;
  float n_scint, n_det, n_out, abs_length, scat_length;
  uint32_t surface;
  float reflectivity;
  uint32_t source;
  float src_x, src_y, src_z, tau;
  uint32_t max_steps;
  uint64_t seed;
};
static_assert(sizeof(Params) == 72, "SimParams layout");

// Optional per-face override: surface model and reflectivity of faces 0..4
// (face 5, the readout, is always the Fresnel interface to n_det).
struct Faces {
  uint32_t surface[6];
  float reflectivity[6];
};

// TallyConfig (include/optphot/transport.hpp:164-168).
struct TallyConfig {
  uint32_t time_bins;
  float time_max;
  uint32_t xy_bins;
};

enum Surface : uint32_t { Polished = 0, Black = 1, Specular = 2, Lambertian = 3 };
enum Fate : uint8_t { Detected = 0, AbsorbedBulk = 1, AbsorbedSurface = 2, Escaped = 3, MaxSteps = 4 };
constexpr int kReadoutFace = 5;  // params.hpp:84
constexpr float kTwoPiF = 6.28318530717958647692f;  // hd.hpp:36
constexpr float kSpeedOfLightF = 299.792458f;       // hd.hpp:37

// ---------------------------------------------------------------------------
// Op counting (Real = Counted). One count per scalar operation of the
// restated source: + - * / compare min max sqrt, one per libm call, and the
// integer work of Philox counted per block (see philox_block below).
struct OpCounter {
  uint64_t fp = 0;     // FP32 add/sub/mul/div/compare/min/max/sqrt/convert
  uint64_t transc = 0; // log / sin / cos / cbrt calls
  uint64_t intop = 0;  // Philox and uniform-conversion integer ops
};
thread_local OpCounter g_ops;

struct Counted {
  float v;
  Counted() : v(0.f) {}
  Counted(float x) : v(x) {}  // NOLINT: implicit on purpose (literals)
};
inline Counted operator+(Counted a, Counted b) { ++g_ops.fp; return a.v + b.v; }
inline Counted operator-(Counted a, Counted b) { ++g_ops.fp; return a.v - b.v; }
inline Counted operator*(Counted a, Counted b) { ++g_ops.fp; return a.v * b.v; }
inline Counted operator/(Counted a, Counted b) { ++g_ops.fp; return a.v / b.v; }
inline Counted operator-(Counted a) { ++g_ops.fp; return -a.v; }
inline bool operator<(Counted a, Counted b) { ++g_ops.fp; return a.v < b.v; }
inline bool operator<=(Counted a, Counted b) { ++g_ops.fp; return a.v <= b.v; }
inline bool operator>(Counted a, Counted b) { ++g_ops.fp; return a.v > b.v; }
inline bool operator>=(Counted a, Counted b) { ++g_ops.fp; return a.v >= b.v; }
inline bool operator==(Counted a, Counted b) { ++g_ops.fp; return a.v == b.v; }
inline bool operator!=(Counted a, Counted b) { ++g_ops.fp; return a.v != b.v; }

// Scalar helpers for each Real.
inline float fmin_(float a, float b) { return fminf(a, b); }
inline float fmax_(float a, float b) { return fmaxf(a, b); }
inline float sqrt_(float a) { return sqrtf(a); }
inline float copysign_(float a, float b) { return copysignf(a, b); }
inline double fmin_(double a, double b) { return fmin(a, b); }
inline double fmax_(double a, double b) { return fmax(a, b); }
inline double sqrt_(double a) { return sqrt(a); }
inline double copysign_(double a, double b) { return copysign(a, b); }
inline Counted fmin_(Counted a, Counted b) { ++g_ops.fp; return fminf(a.v, b.v); }
inline Counted fmax_(Counted a, Counted b) { ++g_ops.fp; return fmaxf(a.v, b.v); }
inline Counted sqrt_(Counted a) { ++g_ops.fp; return sqrtf(a.v); }
inline Counted copysign_(Counted a, Counted b) { ++g_ops.fp; return copysignf(a.v, b.v); }
inline float fval(float x) { return x; }
inline float fval(double x) { return static_cast<float>(x); }
inline float fval(Counted x) { return x.v; }

template <class R> inline R infinity_() { return R(std::numeric_limits<float>::infinity()); }
template <> inline double infinity_<double>() { return std::numeric_limits<double>::infinity(); }
template <class R> inline bool is_inf_(R x) { return fval(x) == std::numeric_limits<float>::infinity(); }

// ---------------------------------------------------------------------------
// Philox4x32-10 (philox.hpp:43-76) and the per-photon stream (philox.hpp:97-149).
struct U4 { uint32_t x, y, z, w; };

inline U4 philox_block(U4 c, uint32_t k0, uint32_t k1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
  const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
  for (int r = 0; r < 10; ++r) {
    if (r > 0) { k0 += W0; k1 += W1; }
    const uint64_t p0 = static_cast<uint64_t>(M0) * c.x;
    const uint64_t p1 = static_cast<uint64_t>(M1) * c.z;
    const uint32_t hi0 = static_cast<uint32_t>(p0 >> 32), lo0 = static_cast<uint32_t>(p0);
    const uint32_t hi1 = static_cast<uint32_t>(p1 >> 32), lo1 = static_cast<uint32_t>(p1);
    c = U4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
  }
  // 10 rounds x (2 mul-lo + 2 mul-hi + 4 xor) + 9 x 2 key additions.
  g_ops.intop += 98;
  return c;
}

// (bits >> 8) + 1 times 2^-24: exactly representable, in (0, 1] (philox.hpp:82-84).
inline float u32_to_uniform(uint32_t bits) {
  g_ops.intop += 4;
  return static_cast<float>((bits >> 8) + 1u) * (1.0f / 16777216.0f);
}

// Counter {block, 0, id_lo, id_hi}, key {seed_lo, seed_hi}; 4 words per block.
struct Stream {
  uint32_t k0, k1, id_lo, id_hi;
  uint32_t block = 0, avail = 0;
  U4 buf{0, 0, 0, 0};
  Stream(uint64_t seed, uint64_t id)
      : k0(static_cast<uint32_t>(seed)), k1(static_cast<uint32_t>(seed >> 32)),
        id_lo(static_cast<uint32_t>(id)), id_hi(static_cast<uint32_t>(id >> 32)) {}
  uint32_t next_u32() {
    if (avail == 0) {
      buf = philox_block(U4{block++, 0u, id_lo, id_hi}, k0, k1);
      avail = 4;
    }
    const uint32_t r = buf.x;
    buf.x = buf.y; buf.y = buf.z; buf.z = buf.w;
    --avail;
    return r;
  }
  float uniform() { return u32_to_uniform(next_u32()); }
  uint32_t draws() const { return 4u * block - avail; }
};

// ---------------------------------------------------------------------------
// Math policies (pmath.hpp:62-158).
struct PlatformMath {};
struct PortableMath {};

inline uint32_t fbits(float x) { uint32_t u; std::memcpy(&u, &x, 4); return u; }
inline float bitsf(uint32_t u) { float x; std::memcpy(&x, &u, 4); return x; }

// Portable natural log: x = 2^e m, m in [sqrt(1/2), sqrt(2)), log m = 2 atanh(s),
// s = (m-1)/(m+1), odd series to s^11, ln 2 split hi/lo (pmath.hpp:62-82).
template <class R> R portable_log(R x) {
  const uint32_t bits = fbits(fval(x));
  int e = static_cast<int>((bits >> 23) & 0xffu) - 127;
  R m = bitsf((bits & 0x007fffffu) | 0x3f800000u);
  if (m > R(1.41421356f)) { m = R(0.5f) * m; ++e; }
  const R s = (m - R(1.0f)) / (m + R(1.0f));
  const R s2 = s * s;
  const R poly = R(1.0f) + s2 * (R(1.0f / 3.0f) + s2 * (R(1.0f / 5.0f) + s2 * (R(1.0f / 7.0f) +
                 s2 * (R(1.0f / 9.0f) + s2 * R(1.0f / 11.0f)))));
  const R ln2_hi = R(6.9313812256e-01f), ln2_lo = R(9.0580006145e-06f);
  const R fe = R(static_cast<float>(e));
  return fe * ln2_hi + (R(2.0f) * s * poly + fe * ln2_lo);
}

// Portable sin/cos of 2 pi u: exact quarter-turn reduction, Taylor to x^9 / x^10
// on |x| <= pi/4 (pmath.hpp:87-119).
template <class R> void portable_sincos_turns(R u, R& s, R& c) {
  const R v = R(4.0f) * u;
  R q = R(floorf(fval(v)));
  R r = v - q;
  if (r > R(0.5f)) { r = r - R(1.0f); q = q + R(1.0f); }
  const R x = r * R(1.57079632679489662f);
  const R x2 = x * x;
  const R sp = x * (R(1.0f) + x2 * (R(-1.0f / 6.0f) + x2 * (R(1.0f / 120.0f) +
               x2 * (R(-1.0f / 5040.0f) + x2 * R(1.0f / 362880.0f)))));
  const R cp = R(1.0f) + x2 * (R(-0.5f) + x2 * (R(1.0f / 24.0f) + x2 * (R(-1.0f / 720.0f) +
               x2 * (R(1.0f / 40320.0f) + x2 * R(-1.0f / 3628800.0f)))));
  const int quadrant = static_cast<int>(fval(q)) & 3;
  if (quadrant == 0) { s = sp; c = cp; }
  else if (quadrant == 1) { s = cp; c = -sp; }
  else if (quadrant == 2) { s = -sp; c = -cp; }
  else { s = -cp; c = sp; }
}

// Portable cube root: exponent/3 first guess, 4 Newton steps (pmath.hpp:123-130).
template <class R> R portable_cbrt(R x) {
  R y = bitsf(fbits(fval(x)) / 3u + 0x2a514067u);
  for (int i = 0; i < 4; ++i) y = y - (y * y * y - x) / (R(3.0f) * y * y);
  return y;
}

template <class R, class M> struct Math;
template <> struct Math<float, PlatformMath> {
  static float log(float x) { return logf(x); }
  static void sincos_turns(float u, float& s, float& c) {
    const float phi = kTwoPiF * u;
    s = sinf(phi);
    c = cosf(phi);
  }
  static float cbrt(float x) { return cbrtf(x); }
};
template <> struct Math<float, PortableMath> {
  static float log(float x) { return portable_log(x); }
  static void sincos_turns(float u, float& s, float& c) { portable_sincos_turns(u, s, c); }
  static float cbrt(float x) { return portable_cbrt(x); }
};
template <> struct Math<double, PlatformMath> {
  static double log(double x) { return std::log(x); }
  static void sincos_turns(double u, double& s, double& c) {
    const double phi = 6.283185307179586476925 * u;
    s = std::sin(phi);
    c = std::cos(phi);
  }
  static double cbrt(double x) { return std::cbrt(x); }
};
template <> struct Math<Counted, PlatformMath> {
  static Counted log(Counted x) { ++g_ops.transc; return logf(x.v); }
  static void sincos_turns(Counted u, Counted& s, Counted& c) {
    const Counted phi = Counted(kTwoPiF) * u;
    ++g_ops.transc; s = sinf(phi.v);
    ++g_ops.transc; c = cosf(phi.v);
  }
  static Counted cbrt(Counted x) { ++g_ops.transc; return cbrtf(x.v); }
};

// ---------------------------------------------------------------------------
// Vec3 (vec3.hpp:17-53).
template <class R> struct V3 { R x, y, z; };
template <class R> inline V3<R> operator+(V3<R> a, V3<R> b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
template <class R> inline V3<R> operator-(V3<R> a, V3<R> b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
template <class R> inline V3<R> operator-(V3<R> a) { return {-a.x, -a.y, -a.z}; }
template <class R> inline V3<R> operator*(R s, V3<R> a) { return {s * a.x, s * a.y, s * a.z}; }
template <class R> inline R dot(V3<R> a, V3<R> b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
template <class R> inline R norm(V3<R> a) { return sqrt_(dot(a, a)); }
template <class R> inline V3<R> normalize(V3<R> a) { return (R(1.0f) / norm(a)) * a; }

// Duff et al. branch-free basis (vec3.hpp:35-41).
template <class R> inline void onb(V3<R> n, V3<R>& t1, V3<R>& t2) {
  const R sign = copysign_(R(1.0f), n.z);
  const R a = R(-1.0f) / (sign + n.z);
  const R b = n.x * n.y * a;
  t1 = {R(1.0f) + sign * n.x * n.x * a, sign * b, -sign * n.x};
  t2 = {b, sign + n.y * n.y * a, -n.y};
}

template <class R, class M> inline V3<R> rotate_about(V3<R> axis, R cos_t, R phi_turns) {
  V3<R> t1, t2;
  onb(axis, t1, t2);
  const R sin_t = sqrt_(fmax_(R(0.0f), R(1.0f) - cos_t * cos_t));
  R sp, cp;
  Math<R, M>::sincos_turns(phi_turns, sp, cp);
  const V3<R> d = (sin_t * cp) * t1 + (sin_t * sp) * t2 + cos_t * axis;
  return normalize(d);
}

// ---------------------------------------------------------------------------
// Sampling (sampling.hpp:17-65).
template <class R, class M> inline R sample_exponential(R length, R u) {
  return is_inf_(length) ? infinity_<R>() : -length * Math<R, M>::log(u);
}
template <class R, class M> inline V3<R> sample_isotropic(R u1, R u2) {
  const R cos_t = R(2.0f) * u1 - R(1.0f);
  const R sin_t = sqrt_(fmax_(R(0.0f), R(1.0f) - cos_t * cos_t));
  R sp, cp;
  Math<R, M>::sincos_turns(u2, sp, cp);
  return {sin_t * cp, sin_t * sp, cos_t};
}
template <class R, class M> inline R sample_rayleigh_cos(R u) {
  const R q = R(4.0f) * u - R(2.0f);
  const R s = sqrt_(q * q + R(1.0f));
  const R a = (q >= R(0.0f)) ? Math<R, M>::cbrt(q + s) : R(1.0f) / Math<R, M>::cbrt(s - q);
  return fmin_(R(1.0f), fmax_(R(-1.0f), a - R(1.0f) / a));
}
template <class R> inline R sample_emission_time_ok(R tau) { return tau > R(0.0f) ? R(1.0f) : R(0.0f); }

// ---------------------------------------------------------------------------
// Geometry (geometry.hpp:25-63).
template <class R> struct Hit { R dist; int face; };
template <class R> inline Hit<R> box_exit(V3<R> p, V3<R> d, R hx, R hy, R hz) {
  Hit<R> h{infinity_<R>(), -1};
  if (d.x != R(0.0f)) {
    const bool pos = d.x > R(0.0f);
    const R t = ((pos ? hx : -hx) - p.x) / d.x;
    if (t < h.dist) h = {t, pos ? 1 : 0};
  }
  if (d.y != R(0.0f)) {
    const bool pos = d.y > R(0.0f);
    const R t = ((pos ? hy : -hy) - p.y) / d.y;
    if (t < h.dist) h = {t, pos ? 3 : 2};
  }
  if (d.z != R(0.0f)) {
    const bool pos = d.z > R(0.0f);
    const R t = ((pos ? hz : -hz) - p.z) / d.z;
    if (t < h.dist) h = {t, pos ? 5 : 4};
  }
  h.dist = fmax_(h.dist, R(0.0f));
  return h;
}
template <class R> inline V3<R> face_normal(int face) {
  const R s = (face & 1) ? R(1.0f) : R(-1.0f);
  const int axis = face >> 1;
  return {axis == 0 ? s : R(0.0f), axis == 1 ? s : R(0.0f), axis == 2 ? s : R(0.0f)};
}
template <class R> inline V3<R> snap_to_face(V3<R> p, int face, R hx, R hy, R hz) {
  const R s = (face & 1) ? R(1.0f) : R(-1.0f);
  const int axis = face >> 1;
  return {axis == 0 ? s * hx : fmin_(fmax_(p.x, -hx), hx),
          axis == 1 ? s * hy : fmin_(fmax_(p.y, -hy), hy),
          axis == 2 ? s * hz : fmin_(fmax_(p.z, -hz), hz)};
}

// Fresnel (fresnel.hpp:30-51).
template <class R> inline R fresnel_R(R n1, R n2, R cos_i) {
  if (n1 == n2) return R(0.0f);
  const R eta = n1 / n2;
  const R sin2_t = eta * eta * fmax_(R(0.0f), R(1.0f) - cos_i * cos_i);
  if (sin2_t >= R(1.0f)) return R(1.0f);
  const R cos_t = sqrt_(R(1.0f) - sin2_t);
  const R rs = (n1 * cos_i - n2 * cos_t) / (n1 * cos_i + n2 * cos_t);
  const R rp = (n2 * cos_i - n1 * cos_t) / (n2 * cos_i + n1 * cos_t);
  return R(0.5f) * (rs * rs + rp * rp);
}
template <class R> inline V3<R> reflect(V3<R> d, V3<R> n) { return d - (R(2.0f) * dot(d, n)) * n; }

// ---------------------------------------------------------------------------
// Transport (transport.hpp:29-159).
template <class R> struct State {
  V3<R> pos, dir;
  R t, path;
  uint32_t nb, ns;
};

// Per-photon extras for the adjoint score and for op accounting.
struct Extra {
  float t_emit = 0.f;
  uint32_t n_refl = 0;       // reflections at painted (specular / Lambertian) faces
  uint32_t painted_abs = 0;  // 1 if absorbed at a painted face
};

enum StepKind : int {
  kStart = 0, kAbsorb = 1, kScatter = 2, kReadoutRefl = 3, kDetect = 4, kPolishedRefl = 5,
  kEscape = 6, kBlack = 7, kPaintAbs = 8, kSpecular = 9, kLambert = 10, kNumKinds = 11
};

struct Surf {
  uint32_t model[6];
  float refl[6];
};

inline Surf make_surf(const Params& p, const Faces* f) {
  Surf s;
  for (int i = 0; i < 6; ++i) {
    s.model[i] = f ? f->surface[i] : p.surface;
    s.refl[i] = f ? f->reflectivity[i] : p.reflectivity;
  }
  return s;
}

// A genstep (the package's extension, no reference counterpart): photons start
// uniformly on the segment (x0,y0,z0)-(x1,y1,z1) at time t0 + u (t1 - t0) plus the
// exponential decay time; same 40-byte layout as optx_genstep of include/optx.h.
struct Genstep {
  float x0, y0, z0, t0, x1, y1, z1, t1;
  uint32_t n_photons, event;
};

// Emission (transport.hpp:55-67). source 2 = genstep segment `g` (extension): the
// three position words become the segment fraction, the time fraction and an
// unused word, so the photon draws the same six words as the reference's sources.
template <class R, class M>
inline State<R> start_photon(const Params& p, Stream& rng, Extra& ex, const Genstep* g = nullptr) {
  V3<R> pos;
  R t_start = R(0.0f);
  if (p.source == 0) {
    pos = {R(p.src_x), R(p.src_y), R(p.src_z)};
  } else if (p.source == 1) {
    const R u1 = rng.uniform(), u2 = rng.uniform(), u3 = rng.uniform();
    pos = {R(p.hx) * (R(2.0f) * u1 - R(1.0f)), R(p.hy) * (R(2.0f) * u2 - R(1.0f)),
           R(p.hz) * (R(2.0f) * u3 - R(1.0f))};
  } else {
    const R u1 = rng.uniform(), u2 = rng.uniform();
    (void)rng.uniform();
    pos = {R(g->x0) + u1 * (R(g->x1) - R(g->x0)), R(g->y0) + u1 * (R(g->y1) - R(g->y0)),
           R(g->z0) + u1 * (R(g->z1) - R(g->z0))};
    t_start = R(g->t0) + u2 * R(g->t1 - g->t0);  // dt in float, as the engine uploads it
  }
  const R ua = rng.uniform(), ub = rng.uniform();
  const V3<R> dir = sample_isotropic<R, M>(ua, ub);
  const R ue = rng.uniform();
  R t = R(p.tau) > R(0.0f) ? -R(p.tau) * Math<R, M>::log(ue) : R(0.0f);
  ex.t_emit = fval(t);
  if (p.source == 2) t = t_start + t;
  return {pos, dir, t, R(0.0f), 0u, 0u};
}

// One step; returns true while alive. kind receives the step's event type.
template <class R, class M>
inline bool step_photon(const Params& p, const Surf& sf, Stream& rng, State<R>& s, uint8_t& fate,
                        Extra& ex, int& kind) {
  const R inv_speed = R(p.n_scint) / R(kSpeedOfLightF);
  const R s_abs = sample_exponential<R, M>(R(p.abs_length), R(rng.uniform()));
  const R s_sca = sample_exponential<R, M>(R(p.scat_length), R(rng.uniform()));
  const Hit<R> hit = box_exit(s.pos, s.dir, R(p.hx), R(p.hy), R(p.hz));

  if (s_abs < hit.dist && s_abs <= s_sca) {
    s.pos = s.pos + s_abs * s.dir;
    s.t = s.t + s_abs * inv_speed;
    s.path = s.path + s_abs;
    fate = AbsorbedBulk;
    kind = kAbsorb;
    return false;
  }
  if (s_sca < hit.dist) {
    s.pos = s.pos + s_sca * s.dir;
    s.t = s.t + s_sca * inv_speed;
    s.path = s.path + s_sca;
    const R u1 = rng.uniform(), u2 = rng.uniform();
    s.dir = rotate_about<R, M>(s.dir, sample_rayleigh_cos<R, M>(u1), u2);
    ++s.ns;
    kind = kScatter;
    return true;
  }
  s.pos = snap_to_face(s.pos + hit.dist * s.dir, hit.face, R(p.hx), R(p.hy), R(p.hz));
  s.t = s.t + hit.dist * inv_speed;
  s.path = s.path + hit.dist;
  ++s.nb;
  const V3<R> normal = face_normal<R>(hit.face);
  const R cos_i = dot(s.dir, normal);

  if (hit.face == kReadoutFace) {
    const R refl = fresnel_R(R(p.n_scint), R(p.n_det), cos_i);
    if (R(rng.uniform()) <= refl) {
      s.dir = reflect(s.dir, normal);
      kind = kReadoutRefl;
      return true;
    }
    fate = Detected;
    kind = kDetect;
    return false;
  }
  const uint32_t model = sf.model[hit.face];
  if (model == Polished) {
    const R refl = fresnel_R(R(p.n_scint), R(p.n_out), cos_i);
    if (R(rng.uniform()) <= refl) {
      s.dir = reflect(s.dir, normal);
      kind = kPolishedRefl;
      return true;
    }
    fate = Escaped;
    kind = kEscape;
    return false;
  }
  if (model == Black) {
    fate = AbsorbedSurface;
    kind = kBlack;
    return false;
  }
  if (!(R(rng.uniform()) <= R(sf.refl[hit.face]))) {
    fate = AbsorbedSurface;
    ex.painted_abs = 1;
    kind = kPaintAbs;
    return false;
  }
  ++ex.n_refl;
  if (model == Specular) {
    s.dir = reflect(s.dir, normal);
    kind = kSpecular;
  } else {
    const R u1 = rng.uniform(), u2 = rng.uniform();
    s.dir = rotate_about<R, M>(-normal, sqrt_(u1), u2);
    kind = kLambert;
  }
  return true;
}

struct Result {
  uint8_t fate;
  uint32_t nb, ns;
  float t, x, y, z, path;
  uint32_t draws;
  Extra ex;
};

template <class R, class M>
inline Result transport(const Params& p, const Surf& sf, uint64_t id, const Genstep* g = nullptr) {
  Stream rng(p.seed, id);
  Extra ex;
  State<R> s = start_photon<R, M>(p, rng, ex, g);
  uint8_t fate = MaxSteps;
  int kind = 0;
  for (uint32_t step = 0; step < p.max_steps; ++step) {
    if (!step_photon<R, M>(p, sf, rng, s, fate, ex, kind)) break;
  }
  return {fate, s.nb, s.ns, fval(s.t), fval(s.pos.x), fval(s.pos.y), fval(s.pos.z), fval(s.path),
          rng.draws(), ex};
}

// time_bin / xy_bin (transport.hpp:170-181).
inline uint32_t time_bin(float t, const TallyConfig& c) {
  const float f = t * (static_cast<float>(c.time_bins) / c.time_max);
  return (f >= static_cast<float>(c.time_bins)) ? c.time_bins : static_cast<uint32_t>(f);
}
inline uint32_t xy_bin(float x, float y, const Params& p, const TallyConfig& c) {
  const float nb = static_cast<float>(c.xy_bins);
  const uint32_t ix = static_cast<uint32_t>(fminf((x + p.hx) / (2.0f * p.hx) * nb, nb - 1.0f));
  const uint32_t iy = static_cast<uint32_t>(fminf((y + p.hy) / (2.0f * p.hy) * nb, nb - 1.0f));
  return iy * c.xy_bins + ix;
}

// Tally layout shared with the engine: [5 fates | time_bins+1 | xy_bins^2 | Σnb | Σns].
inline uint64_t tally_len(const TallyConfig& c) {
  return 5ull + c.time_bins + 1 + static_cast<uint64_t>(c.xy_bins) * c.xy_bins + 2;
}
inline void tally_add(uint64_t* T, const Result& r, const Params& p, const TallyConfig& c) {
  ++T[r.fate];
  if (r.fate == Detected) {
    ++T[5 + time_bin(r.t, c)];
    ++T[5 + c.time_bins + 1 + xy_bin(r.x, r.y, p, c)];
  }
  const uint64_t sums = tally_len(c) - 2;
  T[sums] += r.nb;
  T[sums + 1] += r.ns;
}

template <class R, class M>
Result transport_dispatch(const Params& p, const Surf& sf, uint64_t id) {
  return transport<R, M>(p, sf, id);
}

inline Result run_one(int mode, const Params& p, const Surf& sf, uint64_t id,
                      const Genstep* g = nullptr) {
  switch (mode) {
    case 1: return transport<float, PortableMath>(p, sf, id, g);
    case 2: return transport<double, PlatformMath>(p, sf, id, g);
    default: return transport<float, PlatformMath>(p, sf, id, g);
  }
}

}  // namespace oracle

using namespace oracle;

// ---------------------------------------------------------------------------
// C ABI for the tests (ctypes). math_mode: 0 platform libm (the reference's
// default build), 1 portable math (reference built with OPTPHOT_PORTABLE_MATH),
// 2 double-precision transport.
extern "C" {

int oracle_abi_version() { return 3; }

void oracle_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
  const U4 r = philox_block(U4{ctr[0], ctr[1], ctr[2], ctr[3]}, key[0], key[1]);
  out[0] = r.x; out[1] = r.y; out[2] = r.z; out[3] = r.w;
}

void oracle_stream(uint64_t seed, uint64_t id, uint32_t skip, uint32_t n, uint32_t* out) {
  Stream s(seed, id);
  for (uint32_t i = 0; i < skip; ++i) (void)s.next_u32();
  for (uint32_t i = 0; i < n; ++i) out[i] = s.next_u32();
}

float oracle_u32_to_uniform(uint32_t b) { return u32_to_uniform(b); }
float oracle_portable_log(float x) { return portable_log(x); }
void oracle_portable_sincos_turns(float u, float* s, float* c) { portable_sincos_turns(u, *s, *c); }
float oracle_portable_cbrt(float x) { return portable_cbrt(x); }
float oracle_fresnel(float n1, float n2, float cos_i) { return fresnel_R(n1, n2, cos_i); }
float oracle_rayleigh_cos(float u, int mode) {
  return mode == 1 ? sample_rayleigh_cos<float, PortableMath>(u)
                   : sample_rayleigh_cos<float, PlatformMath>(u);
}

// The direction samplers of the transport (sampling.hpp:22-56), for tests:
// kind 0 isotropic (cos theta = 2 u1 - 1, azimuth u2 turns); kind 1 Lambertian
// about the unit axis a (cos theta = sqrt(u1)); kind 2 Rayleigh scattering of
// the unit direction a (cos theta from the Cardano sampler). Platform math.
void oracle_sample_direction(int kind, float u1, float u2, const float* a, float* out) {
  V3<float> d{};
  if (kind == 0) {
    d = sample_isotropic<float, PlatformMath>(u1, u2);
  } else {
    const V3<float> axis{a[0], a[1], a[2]};
    const float ct = kind == 1 ? sqrt_(u1) : sample_rayleigh_cos<float, PlatformMath>(u1);
    d = rotate_about<float, PlatformMath>(axis, ct, u2);
  }
  out[0] = d.x;
  out[1] = d.y;
  out[2] = d.z;
}

// Records for photons first_id .. first_id + n - 1. Any output pointer may be null.
int oracle_records(const Params* p, const Faces* faces, uint64_t n, uint64_t first_id, int mode,
                   int threads, uint8_t* fate, uint32_t* nb, uint32_t* ns, float* t, float* x,
                   float* y, float* z, float* path, uint32_t* draws) {
  const Surf sf = make_surf(*p, faces);
  const int64_t count = static_cast<int64_t>(n);
#pragma omp parallel for schedule(dynamic, 4096) num_threads(threads > 0 ? threads : omp_get_max_threads())
  for (int64_t i = 0; i < count; ++i) {
    const Result r = run_one(mode, *p, sf, first_id + static_cast<uint64_t>(i));
    if (fate) fate[i] = r.fate;
    if (nb) nb[i] = r.nb;
    if (ns) ns[i] = r.ns;
    if (t) t[i] = r.t;
    if (x) x[i] = r.x;
    if (y) y[i] = r.y;
    if (z) z[i] = r.z;
    if (path) path[i] = r.path;
    if (draws) draws[i] = r.draws;
  }
  return 0;
}

// Tally (layout: see tally_len) for photons first_id .. first_id + n - 1; `out`
// is accumulated into (not cleared).
int oracle_tally(const Params* p, const Faces* faces, const TallyConfig* c, uint64_t n,
                 uint64_t first_id, int mode, int threads, uint64_t* out) {
  const Surf sf = make_surf(*p, faces);
  const uint64_t L = tally_len(*c);
  const int64_t count = static_cast<int64_t>(n);
#pragma omp parallel num_threads(threads > 0 ? threads : omp_get_max_threads())
  {
    std::vector<uint64_t> local(L, 0);
#pragma omp for schedule(dynamic, 4096) nowait
    for (int64_t i = 0; i < count; ++i) {
      tally_add(local.data(), run_one(mode, *p, sf, first_id + static_cast<uint64_t>(i)), *p, *c);
    }
#pragma omp critical
    for (uint64_t k = 0; k < L; ++k) out[k] += local[k];
  }
  return 0;
}

// Batched events: event e has params ev[e], photons offsets[e] .. offsets[e+1]-1
// (global ids; the Philox key is ev[e].seed). Tallies are per event, contiguous.
int oracle_batch_tally(const Params* ev, const uint64_t* offsets, uint32_t n_events,
                       const TallyConfig* c, int mode, int threads, uint64_t* out) {
  const uint64_t L = tally_len(*c);
  for (uint32_t e = 0; e < n_events; ++e) {
    oracle_tally(&ev[e], nullptr, c, offsets[e + 1] - offsets[e], offsets[e], mode, threads,
                 out + static_cast<uint64_t>(e) * L);
  }
  return 0;
}

// Gensteps (extension): genstep g of n_gs emits photons with ids first_id +
// (photons of gensteps 0..g-1) + k, with the physics of ev[g.event] (surfaces
// from faces[g.event] when faces is not null) and adds them to that event's
// tally (out: n_events x tally_len, accumulated into). Records (any pointer may
// be null) are written in photon order when fate is not null.
int oracle_genstep_run(const Params* ev, const Faces* faces, uint32_t n_events, const Genstep* gs,
                       uint64_t n_gs, uint64_t first_id, const TallyConfig* c, int mode, int threads,
                       uint64_t* out, uint8_t* fate, uint32_t* nb, uint32_t* ns, float* t, float* x,
                       float* y, float* z, float* path) {
  const uint64_t L = c ? tally_len(*c) : 0;
  uint64_t off = 0;
  for (uint64_t g = 0; g < n_gs; ++g) {
    const Genstep& G = gs[g];
    if (G.event >= n_events) return 1;
    Params p = ev[G.event];
    p.source = 2;
    const Surf sf = make_surf(p, faces ? &faces[G.event] : nullptr);
    const int64_t count = static_cast<int64_t>(G.n_photons);
    const uint64_t base = off;
#pragma omp parallel num_threads(threads > 0 ? threads : omp_get_max_threads())
    {
      std::vector<uint64_t> local(L, 0);
#pragma omp for schedule(dynamic, 1024) nowait
      for (int64_t i = 0; i < count; ++i) {
        const uint64_t k = base + static_cast<uint64_t>(i);
        const Result r = run_one(mode, p, sf, first_id + k, &G);
        if (out) tally_add(local.data(), r, p, *c);
        if (fate) {
          fate[k] = r.fate;
          nb[k] = r.nb;
          ns[k] = r.ns;
          t[k] = r.t;
          x[k] = r.x;
          y[k] = r.y;
          z[k] = r.z;
          path[k] = r.path;
        }
      }
      if (out) {
#pragma omp critical
        for (uint64_t q = 0; q < L; ++q) out[static_cast<uint64_t>(G.event) * L + q] += local[q];
      }
    }
    off += G.n_photons;
  }
  return 0;
}

// Adjoint score terms. For each photon the FP64 score of its history with
// respect to theta = (abs_length, scat_length, reflectivity, tau):
//   S_La  = path / La^2 - [absorbed in bulk] / La          (La finite)
//   S_Ls  = path / Ls^2 - n_scatter / Ls                   (Ls finite)
//   S_R   = n_reflections_at_painted_faces / R - [absorbed at painted face] / (1 - R)
//   S_tau = -1 / tau + t_emit / tau^2                      (tau > 0)
// and the weight w = w_bin[time_bin(t)] + w_det for detected photons, 0 otherwise.
// grad[j] = sum over photons of w * S_j (FP64). Also fills the time histogram
// (time_bins + 1 counts) and the detected count of the same photons.
int oracle_adjoint(const Params* p, const TallyConfig* c, uint64_t n, uint64_t first_id, int mode,
                   int threads, const double* w_bin, double w_det, double* grad,
                   uint64_t* hist, uint64_t* detected) {
  const Surf sf = make_surf(*p, nullptr);
  const int64_t count = static_cast<int64_t>(n);
  const double La = p->abs_length, Ls = p->scat_length, R = p->reflectivity, tau = p->tau;
  const bool la_on = !std::isinf(La), ls_on = !std::isinf(Ls), tau_on = tau > 0.0;
  const int nt = threads > 0 ? threads : omp_get_max_threads();
  std::vector<double> part(static_cast<size_t>(nt) * 4, 0.0);
  std::vector<uint64_t> hpart(static_cast<size_t>(nt) * (c->time_bins + 2), 0);
  // Fixed static partition + fixed-order merge: deterministic for a given thread count.
#pragma omp parallel num_threads(nt)
  {
    const int tid = omp_get_thread_num();
    double g[4] = {0, 0, 0, 0};
    uint64_t* hp = &hpart[static_cast<size_t>(tid) * (c->time_bins + 2)];
#pragma omp for schedule(static)
    for (int64_t i = 0; i < count; ++i) {
      const Result r = run_one(mode, *p, sf, first_id + static_cast<uint64_t>(i));
      if (r.fate != Detected) continue;
      const uint32_t b = time_bin(r.t, *c);
      ++hp[b];
      ++hp[c->time_bins + 1];
      const double w = (w_bin ? w_bin[b] : 0.0) + w_det;
      if (w == 0.0) continue;
      const double path = r.path;
      if (la_on) g[0] += w * (path / (La * La) - (r.fate == AbsorbedBulk ? 1.0 : 0.0) / La);
      if (ls_on) g[1] += w * (path / (Ls * Ls) - static_cast<double>(r.ns) / Ls);
      g[2] += w * (static_cast<double>(r.ex.n_refl) / R - static_cast<double>(r.ex.painted_abs) / (1.0 - R));
      if (tau_on) g[3] += w * (-1.0 / tau + static_cast<double>(r.ex.t_emit) / (tau * tau));
    }
    for (int j = 0; j < 4; ++j) part[static_cast<size_t>(tid) * 4 + j] = g[j];
  }
  for (int j = 0; j < 4; ++j) grad[j] = 0.0;
  for (int t = 0; t < nt; ++t)
    for (int j = 0; j < 4; ++j) grad[j] += part[static_cast<size_t>(t) * 4 + j];
  if (hist) {
    for (uint32_t b = 0; b <= c->time_bins; ++b) hist[b] = 0;
    if (detected) *detected = 0;
    for (int t = 0; t < nt; ++t) {
      const uint64_t* hp = &hpart[static_cast<size_t>(t) * (c->time_bins + 2)];
      for (uint32_t b = 0; b <= c->time_bins; ++b) hist[b] += hp[b];
      if (detected) *detected += hp[c->time_bins + 1];
    }
  }
  return 0;
}

// Per-bin score moments: moments[5 b] = detected photons in arrival-time bin b,
// moments[5 b + 1 + j] = sum over them of S_j (the score terms of
// oracle_adjoint, detected photons only), b = 0 .. time_bins (last = overflow).
int oracle_score_moments(const Params* p, const TallyConfig* c, uint64_t n, uint64_t first_id,
                         int mode, int threads, double* moments) {
  const Surf sf = make_surf(*p, nullptr);
  const int64_t count = static_cast<int64_t>(n);
  const double La = p->abs_length, Ls = p->scat_length, R = p->reflectivity, tau = p->tau;
  const bool la_on = !std::isinf(La), ls_on = !std::isinf(Ls), tau_on = tau > 0.0;
  const int nt = threads > 0 ? threads : omp_get_max_threads();
  const size_t len = static_cast<size_t>(c->time_bins + 1) * 5;
  std::vector<double> part(static_cast<size_t>(nt) * len, 0.0);
#pragma omp parallel num_threads(nt)
  {
    double* m = &part[static_cast<size_t>(omp_get_thread_num()) * len];
#pragma omp for schedule(static)
    for (int64_t i = 0; i < count; ++i) {
      const Result r = run_one(mode, *p, sf, first_id + static_cast<uint64_t>(i));
      if (r.fate != Detected) continue;
      double* mb = m + 5 * static_cast<size_t>(time_bin(r.t, *c));
      mb[0] += 1.0;
      if (la_on) mb[1] += r.path / (La * La);
      if (ls_on) mb[2] += r.path / (Ls * Ls) - static_cast<double>(r.ns) / Ls;
      mb[3] += static_cast<double>(r.ex.n_refl) / R;
      if (tau_on) mb[4] += -1.0 / tau + static_cast<double>(r.ex.t_emit) / (tau * tau);
    }
  }
  for (size_t k = 0; k < len; ++k) moments[k] = 0.0;
  for (int t = 0; t < nt; ++t)
    for (size_t k = 0; k < len; ++k) moments[k] += part[static_cast<size_t>(t) * len + k];
  return 0;
}

// Algorithmic op counts per step kind, over photons first_id .. first_id+n-1
// (single thread). counts[k*4 + {0,1,2,3}] = {steps, fp ops, transcendental, int ops}
// for k in StepKind (kStart counts photon emissions). Philox blocks are charged
// to the step (or start) that triggered them.
int oracle_opcount(const Params* p, const Faces* faces, uint64_t n, uint64_t first_id,
                   uint64_t* counts) {
  const Surf sf = make_surf(*p, faces);
  for (int k = 0; k < kNumKinds * 4; ++k) counts[k] = 0;
  for (uint64_t i = 0; i < n; ++i) {
    Stream rng(p->seed, first_id + i);
    Extra ex;
    g_ops = OpCounter{};
    State<Counted> s = start_photon<Counted, PlatformMath>(*p, rng, ex);
    counts[kStart * 4 + 0] += 1;
    counts[kStart * 4 + 1] += g_ops.fp;
    counts[kStart * 4 + 2] += g_ops.transc;
    counts[kStart * 4 + 3] += g_ops.intop;
    uint8_t fate = MaxSteps;
    for (uint32_t step = 0; step < p->max_steps; ++step) {
      g_ops = OpCounter{};
      int kind = 0;
      const bool alive = step_photon<Counted, PlatformMath>(*p, sf, rng, s, fate, ex, kind);
      counts[kind * 4 + 0] += 1;
      counts[kind * 4 + 1] += g_ops.fp;
      counts[kind * 4 + 2] += g_ops.transc;
      counts[kind * 4 + 3] += g_ops.intop;
      if (!alive) break;
    }
  }
  return 0;
}

}  // extern "C"
