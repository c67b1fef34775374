// optx_device.cuh - device physics of the optx engine (sm_100a).
//
// One photon step of next-event transport in an axis-aligned box, with the
// physics of the reference's include/optphot/transport.hpp:55-145 and the
// random-number layout of include/optphot/philox.hpp:97-149 (paths relative to
// the reference project zmeskma/GPU_Optical_photons). The arithmetic of every
// quantity follows the reference expression for expression, so that a build
// without FMA contraction and with the portable math of pmath.hpp (OPTX_EXACT=1)
// reproduces the reference CPU histories bit for bit; the fast build
// (OPTX_EXACT=0) calls CUDA's logf / sincosf / cbrtf and lets nvcc contract.
//
// What is restructured for the GPU (values unchanged):
//  * Random words come from a two-block window (8 words of the photon's Philox
//    stream, blocks b and b+1). A step reads its 2..5 words at offsets o..o+4
//    of the window with register selects, and the only Philox call site is
//    after the step, when block b has been used up. The reference instead
//    tests for an empty buffer at every draw, so a warp runs Philox once per
//    draw site at which any lane has run dry.
//  * The three outcomes share one move (pos + d * dir) and the two rotations
//    (Rayleigh scatter, Lambertian bounce) and the two Fresnel interfaces
//    (readout, polished) share one code path each, which keeps lanes with
//    different outcomes on the same instructions.
//  * Reflection on an axis-aligned face is the sign flip of one component and
//    cos_i = |dir[axis]|: both are what reflect() / dot() of fresnel.hpp and
//    transport.hpp:105-106 produce bit for bit for a unit axis normal.
//  * Parameters derived from SimParams once on the host (inv_speed, (n1/n2)^2)
//    are computed with the same float operations as the reference.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#ifndef OPTX_EXACT
#define OPTX_EXACT 0
#endif

namespace optx {

// ---------------------------------------------------------------------------
// Parameters as the kernels see them (built by the host from optx_params and
// optx_faces, see capi.cpp: make_dev_params). 112 bytes, 16-byte aligned so
// that a table of them is read with 128-bit loads.
struct __align__(16) DevParams {
  float hx, hy, hz, inv_speed;             // inv_speed = n_scint / c  (transport.hpp:74)
  float n_scint, n_det, n_out, abs_length;
  float scat_length, tau, src_x, src_y;
  float src_z;
  uint32_t surf_bits;                      // 2 bits per face 0..4: Polished/Black/Specular/Lambertian
  uint32_t max_steps;
  uint32_t source;                         // 0 point, 1 uniform in the volume, 2 genstep segment
  float refl0, refl1, refl2, refl3;        // reflectivity of faces 0..4
  float refl4, eta2_det, eta2_out;         // (n_scint/n_det)^2, (n_scint/n_out)^2 (fresnel.hpp:32-33)
  uint32_t key_lo;
  uint32_t key_hi;
  float inv2hx, inv2hy;                    // 1 / (2 hx), 1 / (2 hy) rounded to nearest (xy_bin)
  uint32_t pad2;
};
static_assert(sizeof(DevParams) == 112, "DevParams layout");
// Indexed reads of a record in global memory (face_refl, step_act) rely on these
// runs of consecutive floats: refl0..refl4, (n_det, n_out), (eta2_det, eta2_out).
static_assert(offsetof(DevParams, refl1) == offsetof(DevParams, refl0) + 4 &&
                  offsetof(DevParams, refl2) == offsetof(DevParams, refl0) + 8 &&
                  offsetof(DevParams, refl3) == offsetof(DevParams, refl0) + 12 &&
                  offsetof(DevParams, refl4) == offsetof(DevParams, refl0) + 16,
              "DevParams reflectivities must be consecutive");
static_assert(offsetof(DevParams, n_out) == offsetof(DevParams, n_det) + 4 &&
                  offsetof(DevParams, eta2_out) == offsetof(DevParams, eta2_det) + 4,
              "DevParams readout / outside pairs must be consecutive");

// Device-side structure-of-arrays photon records (29 bytes per photon).
struct DevRecords {
  uint8_t* fate;
  uint32_t* n_boundary;
  uint32_t* n_scatter;
  float *t, *x, *y, *z, *path;
};

enum : uint32_t { kPolished = 0, kBlack = 1, kSpecular = 2, kLambertian = 3 };
enum : uint32_t { kDetected = 0, kAbsorbedBulk = 1, kAbsorbedSurface = 2, kEscaped = 3, kMaxSteps = 4 };
constexpr int kReadoutFace = 5;
constexpr float kInf = __builtin_huge_valf();

// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon et al., SC11), counter {block, 0, id_lo, id_hi},
// key {seed_lo, seed_hi} (philox.hpp:64-76, :86-115). The 32x32->64 products
// map to one wide multiply each; the key schedule is warp-uniform when all
// lanes share a seed.
__device__ __forceinline__ uint4 philox10(uint4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const unsigned long long p0 = static_cast<unsigned long long>(0xD2511F53u) * c.x;
    const unsigned long long p1 = static_cast<unsigned long long>(0xCD9E8D57u) * c.z;
    c = make_uint4(static_cast<uint32_t>(p1 >> 32) ^ c.y ^ k0, static_cast<uint32_t>(p1),
                   static_cast<uint32_t>(p0 >> 32) ^ c.w ^ k1, static_cast<uint32_t>(p0));
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return c;
}

// (bits >> 8) + 1 times 2^-24, in (0, 1], exact (philox.hpp:82-84).
__device__ __forceinline__ float to_uniform(uint32_t bits) {
  return __uint2float_rn((bits >> 8) + 1u) * (1.0f / 16777216.0f);
}

// The photon's random stream as a window of two consecutive Philox blocks.
// Invariant between steps: w[0..3] = block `blk`, w[4..7] = block `blk + 1`,
// next unread word at w[o], o in [0, 3]; so a step can read 5 words.
// draws() = 4 * blk + o is the reference's PhiloxStream::draws().
// The photon id and key are not stored: callers pass them (the key lives in the
// parameters, the id is first id + photon index), which keeps the per-lane state
// at 10 registers.
struct Rng {
  uint32_t w[8];
  uint32_t o, blk;

  // Starts (draws = 0) or resumes the stream of photon `id` after `draws` words
  // (philox.hpp:117-134): blocks draws/4 and draws/4 + 1 fill the window, as two
  // independent Philox chains (instruction-level parallelism: -1 % on the batch,
  // -3 % on the history kernels).
  __device__ __forceinline__ void init(uint64_t id, uint32_t key_lo, uint32_t key_hi,
                                       uint32_t draws) {
    const uint32_t block = draws >> 2;
    const uint32_t lo = static_cast<uint32_t>(id), hi = static_cast<uint32_t>(id >> 32);
    const uint4 b0 = philox10(make_uint4(block, 0u, lo, hi), key_lo, key_hi);
    const uint4 b1 = philox10(make_uint4(block + 1u, 0u, lo, hi), key_lo, key_hi);
    w[0] = b0.x; w[1] = b0.y; w[2] = b0.z; w[3] = b0.w;
    w[4] = b1.x; w[5] = b1.y; w[6] = b1.z; w[7] = b1.w;
    blk = block;
    o = draws & 3u;
  }
  __device__ __forceinline__ uint32_t draws() const { return 4u * blk + o; }

  // Word o + I of the window, I a compile-time index in [0, 4]: three selects.
  template <int I>
  __device__ __forceinline__ uint32_t word() const {
    const uint32_t lo = (o & 1u) ? w[I + 1] : w[I];
    const uint32_t hi = (o & 1u) ? w[I + 3] : w[I + 2];
    return (o & 2u) ? hi : lo;
  }
  template <int I>
  __device__ __forceinline__ float uniform() const { return to_uniform(word<I>()); }

  // Consumes k words; slides the window (one Philox call per block used up).
  __device__ __forceinline__ void advance(uint32_t k, uint64_t id, uint32_t key_lo,
                                          uint32_t key_hi) {
    o += k;
#pragma unroll 1
    while (o >= 4u) {
      w[0] = w[4]; w[1] = w[5]; w[2] = w[6]; w[3] = w[7];
      ++blk;
      const uint4 b = philox10(make_uint4(blk + 1u, 0u, static_cast<uint32_t>(id),
                                          static_cast<uint32_t>(id >> 32)), key_lo, key_hi);
      w[4] = b.x; w[5] = b.y; w[6] = b.z; w[7] = b.w;
      o -= 4u;
    }
  }
};

// ---------------------------------------------------------------------------
// Math policy (pmath.hpp:134-158). Fast: CUDA's library functions. Exact: the
// portable functions built from correctly rounded operations only (the
// reference's pmath.hpp:62-130 methods: atanh series for log, exact quarter-turn
// reduction and Taylor polynomials for sin/cos, Newton iterations for cbrt),
// compiled without FMA contraction.
#if OPTX_EXACT
__device__ __forceinline__ float m_log(float x) {
  const uint32_t bits = __float_as_uint(x);
  int e = static_cast<int>((bits >> 23) & 0xffu) - 127;
  float m = __uint_as_float((bits & 0x007fffffu) | 0x3f800000u);
  if (m > 1.41421356f) {
    m = 0.5f * m;
    ++e;
  }
  const float s = (m - 1.0f) / (m + 1.0f);
  const float s2 = s * s;
  const float poly = 1.0f + s2 * (1.0f / 3.0f + s2 * (1.0f / 5.0f + s2 * (1.0f / 7.0f +
                     s2 * (1.0f / 9.0f + s2 * (1.0f / 11.0f)))));
  const float fe = static_cast<float>(e);
  return fe * 6.9313812256e-01f + (2.0f * s * poly + fe * 9.0580006145e-06f);
}
__device__ __forceinline__ void m_sincos_turns(float u, float& s, float& c) {
  const float v = 4.0f * u;
  float q = floorf(v);
  float r = v - q;
  if (r > 0.5f) {
    r -= 1.0f;
    q += 1.0f;
  }
  const float x = r * 1.57079632679489662f;
  const float x2 = x * x;
  const float sp = x * (1.0f + x2 * (-1.0f / 6.0f + x2 * (1.0f / 120.0f +
                   x2 * (-1.0f / 5040.0f + x2 * (1.0f / 362880.0f)))));
  const float cp = 1.0f + x2 * (-0.5f + x2 * (1.0f / 24.0f + x2 * (-1.0f / 720.0f +
                   x2 * (1.0f / 40320.0f + x2 * (-1.0f / 3628800.0f)))));
  const int quadrant = static_cast<int>(q) & 3;
  const float ss = (quadrant & 1) ? cp : sp;
  const float cc = (quadrant & 1) ? sp : cp;
  s = (quadrant & 2) ? -ss : ss;
  c = ((quadrant + 1) & 2) ? -cc : cc;
}
__device__ __forceinline__ float m_cbrt(float x) {
  float y = __uint_as_float(__float_as_uint(x) / 3u + 0x2a514067u);
#pragma unroll
  for (int i = 0; i < 4; ++i) y = y - (y * y * y - x) / (3.0f * y * y);
  return y;
}
#else
__device__ __forceinline__ float m_log(float x) { return logf(x); }
__device__ __forceinline__ void m_sincos_turns(float u, float& s, float& c) {
  sincosf(6.28318530717958647692f * u, &s, &c);
}
__device__ __forceinline__ float m_cbrt(float x) { return cbrtf(x); }
#endif

// ---------------------------------------------------------------------------
struct Photon {
  float px, py, pz, dx, dy, dz, t, path;
  uint32_t nb, ns;
};

// Per-photon counters needed by the adjoint's score terms.
struct ScoreAux {
  uint32_t n_refl;  // reflections at painted (specular / Lambertian) faces
  float t_emit;     // sampled emission time
};

// GP: P is a record in global memory, where an indexed load costs one
// instruction; a kernel parameter is read with selects instead (indexing it
// would copy the parameters to local memory).
template <bool GP>
__device__ __forceinline__ float face_refl(const DevParams& P, int face) {
  if (GP) return (&P.refl0)[face];
  float r = P.refl0;
  r = (face == 1) ? P.refl1 : r;
  r = (face == 2) ? P.refl2 : r;
  r = (face == 3) ? P.refl3 : r;
  r = (face == 4) ? P.refl4 : r;
  return r;
}

// Branch-free orthonormal basis (Duff et al., JCGT 6(1) 2017) and rotation
// about `axis` by polar cosine ct and azimuth 2 pi * phi_u (vec3.hpp:35-53).
__device__ __forceinline__ void rotate_about(float ax, float ay, float az, float ct, float phi_u,
                                             float& ox, float& oy, float& oz) {
  const float sign = copysignf(1.0f, az);
  const float a = -1.0f / (sign + az);
  const float b = ax * ay * a;
  const float t1x = 1.0f + sign * ax * ax * a, t1y = sign * b, t1z = -sign * ax;
  const float t2x = b, t2y = sign + ay * ay * a, t2z = -ay;
  const float st = sqrtf(fmaxf(0.0f, 1.0f - ct * ct));
  float sp, cp;
  m_sincos_turns(phi_u, sp, cp);
  const float A = st * cp, B = st * sp;
  const float x = A * t1x + B * t2x + ct * ax;
  const float y = A * t1y + B * t2y + ct * ay;
  const float z = A * t1z + B * t2z + ct * az;
  const float inv = 1.0f / sqrtf(x * x + y * y + z * z);
  ox = inv * x;
  oy = inv * y;
  oz = inv * z;
}

// Rayleigh polar cosine by Cardano inversion of F(mu) = (mu^3 + 3 mu + 4) / 8
// (sampling.hpp:39-44).
__device__ __forceinline__ float rayleigh_cos(float u) {
  const float q = 4.0f * u - 2.0f;
  const float s = sqrtf(q * q + 1.0f);
  // One cube-root call site: cbrt(q + s) for q >= 0, 1 / cbrt(s - q) otherwise.
  const bool pos = q >= 0.0f;
  const float c = m_cbrt(pos ? q + s : s - q);
  const float a = pos ? c : 1.0f / c;
  return fminf(1.0f, fmaxf(-1.0f, a - 1.0f / a));
}

// Unpolarised Fresnel reflectance from n1 into n2 (fresnel.hpp:30-46);
// eta2 = (n1 / n2)^2 precomputed with the same float operations.
__device__ __forceinline__ float fresnel_R(float n1, float n2, float eta2, float cos_i) {
  if (n1 == n2) return 0.0f;
  const float sin2_t = eta2 * fmaxf(0.0f, 1.0f - cos_i * cos_i);
  if (sin2_t >= 1.0f) return 1.0f;
  const float cos_t = sqrtf(1.0f - sin2_t);
  const float rs = (n1 * cos_i - n2 * cos_t) / (n1 * cos_i + n2 * cos_t);
  const float rp = (n2 * cos_i - n1 * cos_t) / (n2 * cos_i + n1 * cos_t);
  return 0.5f * (rs * rs + rp * rp);
}

// Emission (transport.hpp:55-67): position (3 draws, volume source only),
// isotropic direction (2), exponential emission time (1).
//
// Genstep segments (source 2, an extension with no reference counterpart): the
// photon starts at src + u1 (end - src) on the segment from src to end and at
// time t0 + u2 dt + the exponential decay time; u3 is drawn and unused, so the
// photon consumes the same six words as the reference's sources. `seg` holds
// (end x, y, z, t0) and (dt, -, -, -) of the photon's genstep (null otherwise).
constexpr uint32_t kSourceSegment = 2u;

template <bool AUX>
__device__ __forceinline__ void start_photon(const DevParams& P, Photon& s, Rng& r, uint64_t id,
                                             ScoreAux& aux, const float4* seg = nullptr) {
  uint32_t k;
  float t_start = 0.0f;
  if (P.source == 0u) {
    s.px = P.src_x;
    s.py = P.src_y;
    s.pz = P.src_z;
    k = 3u;
  } else if (P.source == 1u) {
    const float u1 = r.uniform<0>(), u2 = r.uniform<1>(), u3 = r.uniform<2>();
    s.px = P.hx * (2.0f * u1 - 1.0f);
    s.py = P.hy * (2.0f * u2 - 1.0f);
    s.pz = P.hz * (2.0f * u3 - 1.0f);
    r.o += 3u;  // o stays <= 3: the window still holds the next 5 words
    k = 3u;
  } else {
    const float4 e = seg[0], w = seg[1];
    const float u1 = r.uniform<0>(), u2 = r.uniform<1>();
    s.px = P.src_x + u1 * (e.x - P.src_x);
    s.py = P.src_y + u1 * (e.y - P.src_y);
    s.pz = P.src_z + u1 * (e.z - P.src_z);
    t_start = e.w + u2 * w.x;
    r.o += 3u;
    k = 3u;
  }
  const float ua = r.uniform<0>(), ub = r.uniform<1>(), ue = r.uniform<2>();
  const float ct = 2.0f * ua - 1.0f;
  const float st = sqrtf(fmaxf(0.0f, 1.0f - ct * ct));
  float sp, cp;
  m_sincos_turns(ub, sp, cp);
  s.dx = st * cp;
  s.dy = st * sp;
  s.dz = ct;
  s.t = P.tau > 0.0f ? -P.tau * m_log(ue) : 0.0f;
  if (AUX) aux.t_emit = s.t;
  if (P.source == kSourceSegment) s.t = t_start + s.t;
  s.path = 0.0f;
  s.nb = 0u;
  s.ns = 0u;
  r.advance(k, id, P.key_lo, P.key_hi);
}

// A step's interaction, decided by step_move: a face index 0..5 (a boundary
// hit), kHitScatter or kHitAbsorb.
constexpr int kHitScatter = 6;
constexpr int kHitAbsorb = 7;

// First half of a step (transport.hpp:71-97): the exponential absorption and
// scattering distances (window words 0 and 1), the box exit, and the move to the
// nearest of the three. Returns the interaction; the window is not advanced.
__device__ __forceinline__ int step_move(const DevParams& P, Photon& s, const Rng& r) {
  const float u_abs = r.uniform<0>(), u_sca = r.uniform<1>();
  const float s_abs = (P.abs_length == kInf) ? kInf : -P.abs_length * m_log(u_abs);
  const float s_sca = (P.scat_length == kInf) ? kInf : -P.scat_length * m_log(u_sca);

  // Distance to the box exit: per axis only the face the photon moves towards
  // (geometry.hpp:25-46).
  // All three quotients are computed and an axis the photon does not move along
  // is then masked (its quotient, a division by zero, is never used): the same
  // values as skipping it, without a branch per axis.
  float dist = kInf;
  int face = -1;
  {
    const bool pos = s.dx > 0.0f;
    const float tt = ((pos ? P.hx : -P.hx) - s.px) / s.dx;
    if (s.dx != 0.0f && tt < dist) { dist = tt; face = pos ? 1 : 0; }
  }
  {
    const bool pos = s.dy > 0.0f;
    const float tt = ((pos ? P.hy : -P.hy) - s.py) / s.dy;
    if (s.dy != 0.0f && tt < dist) { dist = tt; face = pos ? 3 : 2; }
  }
  {
    const bool pos = s.dz > 0.0f;
    const float tt = ((pos ? P.hz : -P.hz) - s.pz) / s.dz;
    if (s.dz != 0.0f && tt < dist) { dist = tt; face = pos ? 5 : 4; }
  }
  dist = fmaxf(dist, 0.0f);

  const bool absorb = s_abs < dist && s_abs <= s_sca;
  const bool scatter = !absorb && s_sca < dist;
  const float d = absorb ? s_abs : (scatter ? s_sca : dist);
  float nx = s.px + d * s.dx, ny = s.py + d * s.dy, nz = s.pz + d * s.dz;
  if (!absorb && !scatter) {  // snap onto the face plane, clamp in-plane (geometry.hpp:57-63)
    const int axis = face >> 1;
    const float sg = (face & 1) ? 1.0f : -1.0f;
    nx = (axis == 0) ? sg * P.hx : fminf(fmaxf(nx, -P.hx), P.hx);
    ny = (axis == 1) ? sg * P.hy : fminf(fmaxf(ny, -P.hy), P.hy);
    nz = (axis == 2) ? sg * P.hz : fminf(fmaxf(nz, -P.hz), P.hz);
  }
  s.px = nx;
  s.py = ny;
  s.pz = nz;
  s.t = s.t + d * P.inv_speed;
  s.path = s.path + d;
  return absorb ? kHitAbsorb : (scatter ? kHitScatter : face);
}

// Surface model of face `face` (the readout face is always polished).
__device__ __forceinline__ uint32_t face_model(const DevParams& P, int face) {
  return (face == kReadoutFace) ? kPolished : ((P.surf_bits >> (2 * face)) & 3u);
}

// Second half of a step (transport.hpp:98-145): the interaction `hit` at the
// photon's position, then the window advance past the words the step used.
// Returns true while the photon is alive; otherwise `fate` is set and the photon
// sits at its final interaction. The window is advanced only for photons that
// stay alive.
// One exit: every outcome falls through to the shared tail (rotation, flip,
// window advance). With sync_mask != 0 (the lanes of the warp that call this
// step together) the warp reconverges before the advance, so the Philox block
// runs once per warp step for all lanes that need one rather than once per
// divergent group.
template <bool AUX, bool GP = false>
__device__ __forceinline__ bool step_act(const DevParams& P, Photon& s, Rng& r, uint64_t id,
                                         uint32_t& fate, ScoreAux& aux, int hit,
                                         uint32_t sync_mask = 0u) {
  const int face = hit;
  const int axis = face >> 1;
  uint32_t k = 2u;           // words consumed by this step
  bool live = true, rotate = false, flip = false;
  float ax = s.dx, ay = s.dy, az = s.dz, ct = 0.0f, phi_u = 0.0f;
  // The window's words 2..4 as uniforms, once for every outcome (each branch
  // below uses its own subset; measured -2 % on the batch against drawing them
  // inside the divergent branches).
  const float u2 = r.uniform<2>(), u3 = r.uniform<3>(), u4 = r.uniform<4>();
  if (hit == kHitAbsorb) {
    fate = kAbsorbedBulk;
    live = false;
  } else if (hit == kHitScatter) {
    ++s.ns;
    ct = rayleigh_cos(u2);
    phi_u = u3;
    rotate = true;
    k = 4u;
  } else {
    ++s.nb;
    const float cos_i = fabsf(axis == 0 ? s.dx : (axis == 1 ? s.dy : s.dz));
    const uint32_t model = face_model(P, face);
    if (model == kPolished) {
      // Readout face: interface to n_det, transmitted = detected; other faces:
      // interface to n_out, transmitted = escaped (transport.hpp:108-128).
      const bool readout = face == kReadoutFace;
      const int oi = readout ? 0 : 1;
      const float n2 = GP ? (&P.n_det)[oi] : (readout ? P.n_det : P.n_out);
      const float R = fresnel_R(P.n_scint, n2, GP ? (&P.eta2_det)[oi] : (readout ? P.eta2_det : P.eta2_out),
                                cos_i);
      k = 3u;
      if (u2 <= R) {
        flip = true;
      } else {
        fate = readout ? kDetected : kEscaped;
        live = false;
      }
    } else if (model == kBlack) {
      fate = kAbsorbedSurface;
      live = false;
    } else if (!(u2 <= face_refl<GP>(P, face))) {
      // Painted reflector (transport.hpp:133-144): absorbed with 1 - R.
      fate = kAbsorbedSurface;
      live = false;
    } else {
      k = 3u;
      if (AUX) ++aux.n_refl;
      if (model == kSpecular) {
        flip = true;
      } else {
        // Lambertian about the inward normal -n (signed zeros as in -face_normal()).
        const float sg = (face & 1) ? -1.0f : 1.0f;
        ax = (axis == 0) ? sg : -0.0f;
        ay = (axis == 1) ? sg : -0.0f;
        az = (axis == 2) ? sg : -0.0f;
        ct = sqrtf(u3);
        phi_u = u4;
        rotate = true;
        k = 5u;
      }
    }
  }
  if (rotate) {
    rotate_about(ax, ay, az, ct, phi_u, s.dx, s.dy, s.dz);
  }
  if (flip) {
    if (axis == 0) s.dx = -s.dx;
    if (axis == 1) s.dy = -s.dy;
    if (axis == 2) s.dz = -s.dz;
  }
  if (sync_mask != 0u) __syncwarp(sync_mask);
  if (live) r.advance(k, id, P.key_lo, P.key_hi);
  return live;
}

// One step (transport.hpp:71-145): move, then interact.
template <bool AUX, bool GP = false>
__device__ __forceinline__ bool step_photon(const DevParams& P, Photon& s, Rng& r, uint64_t id,
                                            uint32_t& fate, ScoreAux& aux,
                                            uint32_t sync_mask = 0u) {
  const int hit = step_move(P, s, r);
  return step_act<AUX, GP>(P, s, r, id, fate, aux, hit, sync_mask);
}

// Tally binning (transport.hpp:170-181); tscale = time_bins / time_max in float.
__device__ __forceinline__ uint32_t time_bin(float t, float tscale, uint32_t time_bins) {
  const float f = t * tscale;
  return (f >= static_cast<float>(time_bins)) ? time_bins : static_cast<uint32_t>(f);
}
// a / b for 0 <= a <= b from y = 1 / b rounded to nearest: the product and two
// FMA corrections. With y the correctly rounded reciprocal and q1 within an ulp
// of a / b, q1 + (a - b q1) y rounds to the correctly rounded quotient
// (Markstein, IBM J. Res. Dev. 34(1), 1990), so this equals the IEEE division
// a / b whenever a / b does not underflow; checked on B200 against __fdiv_rn
// for every a in [b 2^-100, b] of several divisors and for random (a, b) pairs
// (tests/test_gpu_quotient.py). Here a / b >= 2^-25 or a = 0 (a = x + hx with
// |x| <= hx). Measured: -0.8 % per photon-step on the batch (FAST), -1.6 % (EXACT).
__device__ __forceinline__ float quot_rn(float a, float b, float y) {
  const float q0 = a * y;
  const float q1 = fmaf(fmaf(-q0, b, a), y, q0);
  return fmaf(fmaf(-q1, b, a), y, q1);
}
__device__ __forceinline__ uint32_t xy_bin(float x, float y, const DevParams& P, uint32_t xy_bins) {
  const float nbf = static_cast<float>(xy_bins);
  const uint32_t ix = static_cast<uint32_t>(fminf(quot_rn(x + P.hx, 2.0f * P.hx, P.inv2hx) * nbf, nbf - 1.0f));
  const uint32_t iy = static_cast<uint32_t>(fminf(quot_rn(y + P.hy, 2.0f * P.hy, P.inv2hy) * nbf, nbf - 1.0f));
  return iy * xy_bins + ix;
}

}  // namespace optx
