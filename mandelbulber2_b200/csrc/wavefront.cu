// wavefront.cu - the batched wavefront form, with FP32 or FP64 iteration.
//
// A frame (or a batch of frames of uneven size) is rendered as a short
// pipeline of persistent kernels, each over a homogeneous task space:
//
//   stage P  one task per pixel:  the primary march + binary refinement
//            (cRenderWorker::RayMarching, src/render_worker.cpp:708-951);
//            misses are written out, hits are appended to a compact hit list
//   stage N  one task per hit:    the six central-difference DE samples of
//            CalculateNormals (src/shader_calculate_normals.cpp:40-125) and
//            the Lambert term of LightShading (src/shader_light_shading.cpp:61-72)
//   stage D  one thread per stage-S task: AO directions and start records
//   stage S  (1 + ao_rays) tasks per hit: the hard AuxShadow march
//            (src/shader_aux_shadow.cpp:94-321) and one AmbientOcclusion
//            march per AO direction (src/shader_ambient_occlusion.cpp:60-110)
//   stage F  one thread per hit: colour, 8-bit conversion, outputs
//
// Every march is a stream of distance requests p = origin + dir * t.  In
// stages P, N and S each lane holds one task; it runs 2 to 12 formula
// iterations (by formula) between warp votes and, once at most k lanes of the warp are still
// iterating, the lanes whose estimate is done take their march step and
// start their next request, or take the next task from the warp's share of
// the stage's queue (a chunk of tasks per atomicAdd on the stage's counter).  Because a warp only ever runs one
// kind of march, those steps stay converged and cheap, and divergent orbit
// lengths and march lengths cost only the k-lane wait.  A batch walks a job
// table (per-job camera, image size and formula parameters) with the same
// stages, captured once into a CUDA graph.
//
// Two precision policies share the stages:
//   Prec32  the formula iteration in FP32 (fast_formula.cuh) with the ray
//           origin, t and the refinement in FP64;
//   Prec64  the formula iteration in FP64 in the reference's operation order
//           (de_core.cuh) with the march arithmetic of the plain FP64 kernel.
// FP32 points resolve distances down to about 2^-24 of their coordinates;
// where the hit threshold of a view is not well above that (deep zooms, a
// camera inside the solid) the FP32 estimate is noise at the scale the march
// needs.  MBR_ENGINE_WAVEFRONT_AUTO chooses the policy per frame (per job in a
// batch) from the distance estimate at the camera: no ray meets the surface
// closer than that distance, so DE(camera) * threshold-per-unit-distance
// bounds the smallest hit threshold of the view from below.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "de_core.cuh"
#include "fast_formula.cuh"
#include "fastdiv.h"
#include "mbr_internal.h"
#include "pixel_ops.cuh"

namespace mbr {

// formula kinds of the iteration switch
enum { FK_ANY = 0, FK_BULB = 2, FK_MENGER = 7, FK_BOX = 8, FK_BOX_SIMPLE = 108 };

// Views whose smallest hit threshold is below this many FP32 units (2^-24)
// of the camera coordinates iterate in FP64 under MBR_ENGINE_WAVEFRONT_AUTO.
// The FP32 depth error grows about as 0.01 / (threshold in FP32 units); 256
// keeps it near 1e-4 relative at the 99th percentile.
const double kWideRatio = 256.0;

// One render job of a launch: its camera, image size and place in the queue.
struct WJob {
  double cam[3];
  double mrot[9];
  int32_t mrot_zero;
  int32_t width, height, tiles_x;
  int32_t row0, rows;      // the job renders rows [row0, row0 + rows) of its frame
  int32_t persp;           // mbr_projection
  int32_t legacy_y;        // legacy coordinate system (image y flipped)
  long long first;         // first work item of this job in the pixel queue
  long long pixel_offset;  // first pixel of this job in the outputs
  double fov, aspect;
  double resolution, detail;  // CalcDistThresh factors (1/height, detail level)
  float c0;                // threshold per unit distance: resolution * fov / detail (halved: equirectangular)
  float fovf;              // AO end distance per unit distance: fov (halved: equirectangular)
  float cthr;              // constant threshold (halved: equirectangular)
  FastDiv div_w, div_tx;   // divisions by width and tiles_x
};

// A surface hit, produced by stage P and completed by stages N and S.
struct HitRec {
  double px, py, pz;  // hit point
  double depth;       // scan distance t of the hit
  double thr;         // distThresh at the hit
  long long pix;      // output index
  int iters;          // iters of the last primary DE evaluation
  float nx, ny, nz;   // normal
  float shade;        // Lambert term before the shadow
  float shadow;       // AuxShadow result
  int job;
  unsigned int ray;   // pixel index within its job (RNG streams)
  // sum of the AO march results in 32.32 fixed point: integer atomics make
  // the sum independent of the order in which the AO marches finish
  unsigned long long ao_q;
};

__device__ __forceinline__ void ao_add(HitRec *r, double s) {
  atomicAdd(&r->ao_q, (unsigned long long)(s * 4294967296.0));
}

// Device-side counters of one launch (in the context's scratch).
struct Counters4 {
  unsigned long long pixels_next;  // stage P queue
  unsigned long long hits;         // hits appended by stage P
  unsigned long long normals_next; // stage N queue
  unsigned long long shade_next;   // stage S queue
};

// FP64 parameters of a non-hybrid formula: the slot's double parameters, read
// by the reference-order formulas of de_core.cuh, and the Compute settings.
struct WideParams {
  DevSlot slot;
  int formula, maxN, de_fn, min_n;
  int julia, add_c, check_bailout, box_simple;  // box_simple: as FastParams::box_simple
  double bailout;
  double jc[3];  // julia_c * fractal_constant_factor
  double cm[3];  // fractal_constant_factor
  // simple Mandelbox: folding limit, fR2, fR2/mR2, scale, |scale|, bailout^2
  double lim, fr2, fmx, scale, ascale, bailout2;
  MbRot rot;  // Mandelbox rotations (the simple form is off when any is on)
};

__host__ __device__ inline WideParams load_wide_params(const DevScene &sc) {
  WideParams w;
  w.slot = sc.slot[0];
  w.formula = sc.slot[0].formula;
  w.maxN = sc.formula_maxiter;
  w.de_fn = sc.de_analytic;
  w.min_n = sc.min_n;
  w.julia = sc.julia;
  w.add_c = sc.slot[0].add_c;
  w.check_bailout = sc.slot[0].check_bailout;
  w.bailout = sc.slot[0].d[P_BAILOUT];
  for (int k = 0; k < 3; k++) {
    w.jc[k] = sc.julia_c[k] * sc.cmul[k];
    w.cm[k] = sc.cmul[k];
  }
  const DevSlot &s = sc.slot[0];
  const double L = s.d[P_MB_LIMIT], F = s.d[P_MB_FACTOR1];
  w.rot = sc.mbrot;
  w.box_simple = (s.formula == MBR_FORMULA_MANDELBOX && s.d[P_MB_VALUE] == 2.0 * L && L > 0.0 && F > 1.0 &&
                  !s.has_offset && !sc.mbrot.folds && !sc.mbrot.main) ? 1 : 0;
  w.lim = L;
  w.fr2 = s.d[P_MB_FR2];
  w.fmx = F;
  w.scale = s.d[P_MB_SCALE];
  w.ascale = s.d[P_MB_ABS_SCALE];
  w.bailout2 = w.bailout * w.bailout;
  return w;
}

struct Launch {
  const WJob *jobs;        // njobs entries (device)
  const FastParams *fps;   // per job (device), FP32 policy
  const WideParams *wps;   // per job (device), FP64 policy
  int njobs;
  long long total;         // pixel work items
  HitRec *hits;            // capacity: total
  float4 *sorg;            // per hit: FP32 hit point and threshold (stage S origins)
  float4 *sdir;            // per stage-S task: direction and end (w < 0: shadow, w == 0: no march)
  Counters4 *ctr;
  const int *gate;         // MBR_ENGINE_WAVEFRONT_AUTO: the policy flag; null: always run
  int gate_value;          // the flag value this pipeline runs under (0 FP32, 1 FP64)
  int refill_k;
  int layout;
  int ao_rays;             // AO tasks per hit (1 for fast AO)
  int ao_fast;             // fast AO: the AO task samples along the normal
  int shadow_tasks;        // 1 when the shadow march runs (shading && shadow)
  int want_normal;
  FastDiv div_per;         // division by shadow_tasks + ao_rays (set by launch_pipeline)
  // GI frames
  double *path_rad;              // radiance of every path of the launch
  HitRec *hits_next;             // the next level's vertex list
  unsigned long long *next_hits; // its counter
  FastDiv div_spp;               // division by samples per pixel
  int level;                     // bounce level of the vertex list in `hits`
  int row0;                      // first row of the launch
  int normal_slot;               // stats counter of stage N (K_NORMAL; K_GI in GI frames)
};

// Stage-S AO tasks per hit: the AO marches, or the one fast-AO task.
static inline int ao_tasks(const DevFrame &fr) { return fr.ao_fast ? 1 : fr.ao_rays; }

// True when this pipeline's kernels have nothing to do (the other precision
// renders the frame).
__device__ __forceinline__ bool gated_off(const Launch &L) { return L.gate && *L.gate != L.gate_value; }

__device__ __forceinline__ int job_of(const WJob *jobs, int n, long long idx) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (jobs[mid].first <= idx) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

__host__ __device__ inline int fast_kind(const FastParams &f) {
  if (f.formula == MBR_FORMULA_MANDELBOX) return f.box_simple ? FK_BOX_SIMPLE : FK_BOX;
  if (f.formula == MBR_FORMULA_MANDELBULB) return FK_BULB;
  return FK_MENGER;
}

__host__ __device__ inline int wide_kind(const WideParams &w) {
  if (w.formula == MBR_FORMULA_MANDELBOX) return w.box_simple ? FK_BOX_SIMPLE : FK_BOX;
  if (w.formula == MBR_FORMULA_MANDELBULB) return FK_BULB;
  return FK_MENGER;
}

__device__ __forceinline__ float fmadd(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double fmadd(double a, double b, double c) { return fma(a, b, c); }

// Formula iterations between warp votes.  A vote (active mask, ballot, count)
// costs a few instructions per lane; orbits of the folding formulas run 7-19
// iterations per estimate, so a vote every 12 is cheap against the wait it
// causes (measured on the 1080p Mandelbox: 2 -> 7.5 ms, 6 -> 6.4 ms,
// 12 -> 6.3 ms per frame), while the Mandelbulb's 1-3 iterations per
// estimate at the usual views want a vote every 2.
template <int FK>
struct kVoteEvery {
  static constexpr int n = (FK == FK_BULB) ? 2 : ((FK == FK_ANY) ? 4 : 12);
};

// True when more than k bits of m are set.  k <= 2 takes the lowest set bit
// off on the ALU pipe instead of a POPC on the (eighth-rate) XU pipe.
__device__ __forceinline__ bool more_than(unsigned m, int k) {
  if (k == 0) return m != 0u;
  if (k == 1) return (m & (m - 1u)) != 0u;
  if (k == 2) {
    const unsigned a = m & (m - 1u);
    return (a & (a - 1u)) != 0u;
  }
  return __popc(m) > k;
}

// ============================================================================
// Precision policies: the per-lane state of one distance estimate, its
// start, one formula iteration and the final distance.
// ============================================================================
struct Prec32 {
  typedef float D;  // distance and threshold arithmetic of the march
  typedef FastParams Params;
  enum { kWide = 0, kHyb = 0 };
  struct State {
    Z3 z, c;
    float dr, r2;
    int it;
  };
  __host__ __device__ static int kind(const Params &f) { return fast_kind(f); }
  __device__ static const Params &job_params(const Launch &L, int job) { return L.fps[job]; }

  __device__ static void start(State &e, const Params &fp, float qx, float qy, float qz) {
    e.z.x = qx;
    e.z.y = qy;
    e.z.z = qz;
    if (!fp.add_c) e.c = Z3{0.f, 0.f, 0.f};
    else if (fp.julia) e.c = Z3{fp.jc_x, fp.jc_y, fp.jc_z};
    else e.c = Z3{qx * fp.cm_x, qy * fp.cm_y, qz * fp.cm_z};
    e.dr = 1.f;
    e.it = 0;
    e.r2 = fmaf(qx, qx, fmaf(qy, qy, qz * qz));
  }
  __device__ static void start(State &e, const Params &fp, double qx, double qy, double qz) {
    start(e, fp, float(qx), float(qy), float(qz));
  }

  // One iteration; false once the orbit is done (bailout or maxN).
  template <int FK>
  __device__ static bool step(int kind, State &e, const Params &fp) {
    const int k = (FK == FK_ANY) ? kind : FK;
    if (k == FK_BOX_SIMPLE) it_mandelbox<true>(e.z, e.dr, e.c, fp);
    else if (k == FK_BOX) it_mandelbox<false>(e.z, e.dr, e.c, fp);
    else if (k == FK_BULB) it_mandelbulb(e.z, e.dr, e.c, fp, sqrtf(e.r2));
    else it_menger(e.z, e.dr, e.c, fp);
    e.it++;
    e.r2 = fmaf(e.z.x, e.z.x, fmaf(e.z.y, e.z.y, e.z.z * e.z.z));
    return e.r2 <= fp.bailout2 && e.it < fp.maxN;
  }

  __device__ static float distance(const State &e, const Params &fp, float detail, int &iters) {
    iters = (e.r2 > fp.bailout2) ? e.it : e.it + 1;
    return final_de(fp, e.r2, e.dr, iters, detail);
  }
};

struct Prec64 {
  typedef double D;
  typedef WideParams Params;
  enum { kWide = 1, kHyb = 0 };
  struct State {
    double zx, zy, zz, cx, cy, cz, dr, r;
    int it, brk;  // iterations done; 1 when the loop ended by a break (bailout or NaN)
  };
  __host__ __device__ static int kind(const Params &w) { return wide_kind(w); }
  __device__ static const Params &job_params(const Launch &L, int job) { return L.wps[job]; }

  // Compute's start (compute_fractal.cpp:74-130): z = c = the point, DE = 1
  __device__ static void start(State &e, const Params &, double qx, double qy, double qz) {
    e.zx = qx;
    e.zy = qy;
    e.zz = qz;
    e.cx = qx;
    e.cy = qy;
    e.cz = qz;
    e.dr = 1.0;
    e.r = len4<double, false>(V4<double>{qx, qy, qz, 0.0});
    e.it = 0;
    e.brk = 0;
  }

  // One pass of the Compute loop body for a non-hybrid scene, as
  // calc_distance<double, F, false> runs it (compute_fractal.cpp:170-321).
  // The simple Mandelbox (folding value 2 * limit, no offset) runs the fold
  // rewrites of fast_formula.cuh in FP64: box fold 2 clamp(z, -L, L) - z,
  // sphere-fold factor clamp(fR2 / r2, 1, fR2 / mR2) with a correctly rounded
  // reciprocal, scale and c-addition fused, bailout tested on |z|^2 and |z|
  // taken once when the orbit ends; the result differs from the reference's
  // operation order in the last bits only.
  template <int FK>
  __device__ static bool step(int kind, State &e, const Params &fp) {
    const int k = (FK == FK_ANY) ? kind : FK;
    if (k == FK_BOX_SIMPLE) {
      const double L = fp.lim;
      const double x = fma(2.0, fmin(fmax(e.zx, -L), L), -e.zx);
      const double y = fma(2.0, fmin(fmax(e.zy, -L), L), -e.zy);
      const double z = fma(2.0, fmin(fmax(e.zz, -L), L), -e.zz);
      const double r2 = fma(x, x, fma(y, y, z * z));
      const double fs = fmin(fmax(fp.fr2 * __drcp_rn(r2), 1.0), fp.fmx);
      const double s = fs * fp.scale;
      e.dr = fma(e.dr, fs * fp.ascale, 1.0);
      double ax = 0.0, ay = 0.0, az = 0.0;
      if (fp.add_c) {
        if (fp.julia) {
          ax = fp.jc[0];
          ay = fp.jc[1];
          az = fp.jc[2];
        } else {
          ax = e.cx * fp.cm[0];
          ay = e.cy * fp.cm[1];
          az = e.cz * fp.cm[2];
        }
      }
      e.zx = fma(x, s, ax);
      e.zy = fma(y, s, ay);
      e.zz = fma(z, s, az);
      e.it++;
      const double rr = fma(e.zx, e.zx, fma(e.zy, e.zy, e.zz * e.zz));
      if (!(rr <= fp.bailout2) && fp.check_bailout) {
        e.r = sqrt(rr);
        e.brk = 1;
        return false;
      }
      if (e.it >= fp.maxN) {
        e.r = sqrt(rr);
        return false;
      }
      return true;
    }
    V4<double> z{e.zx, e.zy, e.zz, 0.0};
    const V4<double> last = z;
    double de = e.dr;
    if (k == FK_BULB) f_mandelbulb<double>(z, e.r, de, fp.slot);
    else if (k == FK_MENGER) f_menger<double, false>(z, de, fp.slot);
    else f_mandelbox<double, false, true>(z, de, fp.slot, &fp.rot);
    if (fp.add_c) {
      if (fp.julia) {
        z.x = z.x + fp.jc[0];
        z.y = z.y + fp.jc[1];
        z.z = z.z + fp.jc[2];
      } else {
        z.x = z.x + e.cx * fp.cm[0];
        z.y = z.y + e.cy * fp.cm[1];
        z.z = z.z + e.cz * fp.cm[2];
      }
    }
    e.it++;
    e.dr = de;
    if (nan4<double, false>(z)) {  // revert to the last finite orbit point
      e.zx = last.x;
      e.zy = last.y;
      e.zz = last.z;
      e.r = len4<double, false>(last);
      e.brk = 1;
      return false;
    }
    e.zx = z.x;
    e.zy = z.y;
    e.zz = z.z;
    e.r = len4<double, false>(z);
    if (fp.check_bailout && e.r > fp.bailout) {
      e.brk = 1;
      return false;
    }
    return e.it < fp.maxN;
  }

  // Final DE and CalculateDistanceSimple's clamps (compute_fractal.cpp:561-621,
  // calculate_distance.cpp:569, 604-605).
  __device__ static double distance(const State &e, const Params &fp, double detail, int &iters) {
    iters = e.brk ? e.it : e.it + 1;
    const double r = e.r, DE = e.dr;
    double d;
    if (DE > 0.0) {
      if (fp.de_fn == 2) d = (r > 1.0) ? 0.5 * r * log(r) / DE : 0.0;
      else if (fp.de_fn == 1) d = r / DE;
      else if (fp.de_fn == 3) d = (r - 2.0) / DE;
      else d = r;
    } else {
      d = r;
    }
    if (iters < fp.min_n && d < detail) d = detail;
    if (d < 0.0) d = 0.0;
    if (d > 10.0) d = 10.0;
    return d;
  }
};

// Hybrid sequences (single-frame launches): the FP32 iteration of
// calc_distance<float, 0, false> one pass at a time - the slot of iteration
// i from the sequence table (CreateSequence), per-slot formula, c-addition,
// weight blend, NaN revert and per-slot bailout (compute_fractal.cpp:170-321),
// and the hybrid DE function of the final distance (:503-557).  The scene
// lives in device memory (the launch scratch) and is read through a pointer.
struct HybParams {
  const DevScene *sc;
};

// EXT: every formula and the Mandelbox rotations (scene_extended scenes);
// hybrids of the three specialised formulas use the lighter PrecHyb.
template <bool EXT>
struct PrecHybT {
  typedef float D;
  typedef HybParams Params;
  enum { kWide = 0, kHyb = 1 };
  struct State {
    float zx, zy, zz, cx, cy, cz, dr, r;
    int it, brk;
  };
  __host__ __device__ static int kind(const Params &) { return FK_ANY; }

  __device__ static void start(State &e, const Params &, float qx, float qy, float qz) {
    e.zx = qx;
    e.zy = qy;
    e.zz = qz;
    e.cx = qx;
    e.cy = qy;
    e.cz = qz;
    e.dr = 1.0f;
    e.r = len4<float, false>(V4<float>{qx, qy, qz, 0.0f});
    e.it = 0;
    e.brk = 0;
  }
  __device__ static void start(State &e, const Params &fp, double qx, double qy, double qz) {
    start(e, fp, float(qx), float(qy), float(qz));
  }

  template <int FK>
  __device__ static bool step(int, State &e, const Params &fp) {
    const DevScene &sc = *fp.sc;
    const int i = e.it;
    const int k = (i < sc.length) ? int(sc.seq[i]) : int(sc.seq[0]);
    const DevSlot &s = sc.slot[k];
    V4<float> z{e.zx, e.zy, e.zz, 0.0f};
    const V4<float> last = z;
    float de = e.dr;
    if (EXT) global_folds<float, false>(sc, z, e.r, de);
    const V4<float> tempZ = z;
    const float tempDE = de;
    // the Aexion, the one formula that replaces c, is 4-D and never runs here
    V4<float> c{e.cx, e.cy, e.cz, 0.0f};
    AuxX<float> ax{1.0f, 0.0f, 0.0f, 1.0f, 1000.0f, c};  // formulas with orbit state do not run here (check_supported)
    if (s.d[P_WEIGHT] > 0.0) formula_dispatch<float, false, EXT>(s.formula, z, e.r, de, s, &sc.mbrot, &sc.ifs, i, c, ax);
    if (s.add_c) {
      if (sc.julia) {
        z.x = z.x + juliac_of<float>(sc, 0);
        z.y = z.y + juliac_of<float>(sc, 1);
        z.z = z.z + juliac_of<float>(sc, 2);
      } else {
        z.x = z.x + e.cx * cmul_of<float>(sc, 0);
        z.y = z.y + e.cy * cmul_of<float>(sc, 1);
        z.z = z.z + e.cz * cmul_of<float>(sc, 2);
      }
    }
    if (sc.is_hybrid) {
      const double kw = s.d[P_WEIGHT];
      if (kw < 1.0) {
        z = smooth4<float, false>(tempZ, z, kw);
        de = de * float(kw) + tempDE * float(1.0 - kw);
      }
    }
    e.it = i + 1;
    e.dr = de;
    if (nan4<float, false>(z)) {
      e.zx = last.x;
      e.zy = last.y;
      e.zz = last.z;
      e.r = len4<float, false>(last);
      e.brk = 1;
      return false;
    }
    e.zx = z.x;
    e.zy = z.y;
    e.zz = z.z;
    e.r = len4<float, false>(z);
    if (s.check_bailout && e.r > P<float>(s, P_BAILOUT)) {
      e.brk = 1;
      return false;
    }
    return e.it < sc.formula_maxiter;
  }

  __device__ static float distance(const State &e, const Params &fp, float detail, int &iters) {
    const DevScene &sc = *fp.sc;
    if (EXT && sc.limits) {  // outside the limit box: its distance (the iteration is not used)
      const float lbd = limit_box_distance<float>(sc, e.cx, e.cy, e.cz);
      if (lbd > detail) {
        iters = 0;
        return lbd;
      }
    }
    iters = e.brk ? e.it : e.it + 1;
    float d = final_distance<float, EXT ? F_EXT : 0, false>(sc, V4<float>{e.zx, e.zy, e.zz, 0.0f}, e.r, e.dr);
    if (iters < sc.min_n && d < detail) d = detail;
    if (d < 0.0f) d = 0.0f;
    if (d > 10.0f) d = 10.0f;
    if (EXT) {  // the union with the primitives, at the request point c
      for (int k = 0; k < sc.n_prims; k++) {
        const float pd = prim_distance<float>(sc.prim[k], e.cx, e.cy, e.cz);
        if (pd < d) d = pd;
      }
    }
    return d;
  }
};
typedef PrecHybT<false> PrecHyb;

// ============================================================================
// The persistent skeleton: refill lanes from a task counter, iterate, step.
// Stage provides (Real: the precision of its request points, D: of its distances):
//   bool start(long long task, Real &qx, &qy, &qz)   - first request (false: nothing to march)
//   bool step(D d, int iters, Real &qx, &qy, &qz)    - consume a result; true: next request
//   const Params &params()  - formula of the current task
//   int kind()              - formula kind (FK_ANY launches)
//   D detail()              - detail size of the current request
// ============================================================================
// fpk: the formula parameters of a single-job launch, the kernel parameter
// itself, so that the iteration reads its constants as constant-bank operands
// (a copy held in the stage is read through indexed constant loads); batch
// launches (Stage::kMulti) read the per-job copy the stage loads.
template <int FK, class P, class Stage>
__device__ __forceinline__ void run_stage(Stage &S, const typename P::Params &fpk, unsigned long long *counter,
                                          long long total, int refill_k, unsigned int *my_de,
                                          unsigned long long *my_iters) {
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const unsigned lanemask_lt = (1u << lane) - 1u;
  typename P::State e = {};
  bool has = false, iterating = false, drained = false;
  long long q_next = 0, q_end = 0;  // the warp's unstarted tasks [q_next, q_end)
  const long long warps = (long long)gridDim.x * (long long)(blockDim.x >> 5);
  const int chunk = (int)min(64ll, max(1ll, total / (32ll * max(warps, 1ll))));
  unsigned int de_n = 0;
  unsigned long long it_n = 0;
  for (;;) {
    // ---- refill lanes without a task from the warp's share of the queue.
    // A warp takes max(chunk, waiting lanes) tasks per atomic on the stage's
    // counter; chunk grows with the tasks per resident warp (up to 64), so a
    // large queue costs fewer atomics and dependent waits, while a small one
    // keeps its tail balanced.
    unsigned need = __ballot_sync(FULL, !has && !drained);
    while (need) {
      const int waiting = __popc(need);
      if (q_next >= q_end) {
        const int take_n = max(chunk, waiting);
        unsigned long long base = 0ull;
        if (lane == 0) base = atomicAdd(counter, (unsigned long long)take_n);
        base = __shfl_sync(FULL, base, 0);
        if ((long long)base >= total) {
          drained = true;
          break;
        }
        q_next = (long long)base;
        q_end = min((long long)base + take_n, total);
      }
      const int take = (int)min((long long)waiting, q_end - q_next);
      const int rank = __popc(need & lanemask_lt);
      if (((need >> lane) & 1u) && rank < take) {
        typename Stage::Real qx, qy, qz;
        if (S.start(q_next + rank, qx, qy, qz)) {
          P::start(e, Stage::kMulti ? S.params() : fpk, qx, qy, qz);
          has = true;
          iterating = true;
        }
      }
      q_next += take;
      need = __ballot_sync(FULL, !has && !drained);
    }
    if (!__any_sync(FULL, iterating)) break;
    const int k = drained ? 0 : refill_k;
    // ---- formula iterations, kVoteEvery<FK> between votes, until <= k lanes
    // still iterate.  A lane whose orbit ends leaves the loop by a branch, so
    // the remaining lanes run the iteration without select instructions for
    // finished ones; the vote counts the lanes still in the loop.
    const typename P::Params &fp = Stage::kMulti ? S.params() : fpk;
    const int kind = S.kind();
    if (iterating) {
      for (;;) {
        bool ended = false;
#pragma unroll
        for (int u = 0; u < kVoteEvery<FK>::n; u++) {
          if (!P::template step<FK>(kind, e, fp)) {
            ended = true;
            break;
          }
        }
        if (ended) {
          iterating = false;
          break;
        }
        if (!more_than(__ballot_sync(__activemask(), 1), k)) break;
      }
    }
    __syncwarp();
    // ---- lanes whose estimate is done: distance, then the march step
    if (has && !iterating) {
      int iters;
      const typename P::D d = P::distance(e, fp, S.detail(), iters);
      de_n++;
      it_n += (unsigned long long)iters;
      typename Stage::Real qx, qy, qz;
      if (S.step(d, iters, qx, qy, qz)) {
        P::start(e, Stage::kMulti ? S.params() : fpk, qx, qy, qz);
        iterating = true;
      } else {
        has = false;
      }
    }
  }
  *my_de += de_n;
  *my_iters += it_n;
}

// Adds this warp's counts to the launch stats (no block barrier: a warp of a
// persistent CTA leaves as soon as its queue is drained).
__device__ __forceinline__ void flush_counts(const DevOutputs &out, unsigned int my_de, unsigned long long my_iters,
                                             int slot_a, unsigned int val_a, int slot_b, unsigned int val_b) {
  if (!out.stats) return;
  const unsigned FULL = 0xffffffffu;
  unsigned long long *st = reinterpret_cast<unsigned long long *>(out.stats);
  const unsigned de = __reduce_add_sync(FULL, my_de);
  const unsigned a = __reduce_add_sync(FULL, val_a);
  const unsigned b = __reduce_add_sync(FULL, val_b);
  unsigned long long it = my_iters;
  for (int o = 16; o > 0; o >>= 1) it += __shfl_down_sync(FULL, it, o);
  if ((threadIdx.x & 31) == 0) {
    if (de) atomicAdd(st + K_DE, (unsigned long long)de);
    if (a) atomicAdd(st + slot_a, (unsigned long long)a);
    if (b) atomicAdd(st + slot_b, (unsigned long long)b);
    if (it) atomicAdd(st + K_ITERS, it);
  }
}

// ============================================================================
// Stage P: primary march with binary refinement, one task per pixel.
// ============================================================================
template <bool MULTI, class P>
struct PrimaryStage {
  typedef double Real;
  static constexpr bool kMulti = MULTI;
  typedef typename P::D D;
  const DevFrame &fr;
  const Launch &L;
  const DevOutputs &out;
  const WJob *jb;
  typename P::Params fp;
  int kd;
  int job;
  // ray
  double dx, dy, dz, ox, oy, oz, t, stp, dir_len;
  double lx, ly, lz;  // previous request point (dead-ray check)
  D thr, c0, dist_prev, search_limit;
  int phase, sub, count, last_iters;
  unsigned int pm, ray, binary_de;
  long long pix;

  __device__ const typename P::Params &params() const { return fp; }
  __device__ int kind() const { return kd; }
  __device__ D detail() const { return thr; }

  // distThresh at the request point (render_worker.cpp:653-679): FP64 from
  // |camera - q| as the plain kernel computes it; FP32 from t
  // with the tail of thresh_tail: an equirectangular view halves it (in the
  // FP32 form inside c0 and `cthr`), advanced quality clamps it
  __device__ void set_thr(double qx, double qy, double qz) {
    if (P::kWide) {
      double v;
      if (fr.constant_de_threshold) {
        v = fr.de_thresh;
      } else {
        const double ax = jb->cam[0] - qx, ay = jb->cam[1] - qy, az = jb->cam[2] - qz;
        const double l = sqrt(ax * ax + ay * ay + az * az);
        v = l * jb->resolution * jb->fov / jb->detail;
      }
      thr = D(thresh_tail(fr, jb->persp, v));
    } else {
      float v = fr.constant_de_threshold ? jb->cthr : float(t) * float(c0);
      if (fr.adv_quality) {
        if (v > float(fr.detail_size_max)) v = float(fr.detail_size_max);
        if (v < float(fr.detail_size_min)) v = float(fr.detail_size_min);
      }
      thr = D(v);
    }
  }

  __device__ void point(double &qx, double &qy, double &qz) {
    qx = fma(dx, t, ox);
    qy = fma(dy, t, oy);
    qz = fma(dz, t, oz);
    set_thr(qx, qy, qz);
  }

  // The next march point; false when the ray is stuck: the point did not
  // move or is not finite (render_worker.cpp:747-756).
  __device__ bool advance(double &qx, double &qy, double &qz) {
    const double nx = fma(dx, t, ox), ny = fma(dy, t, oy), nz = fma(dz, t, oz);
    if ((nx == lx && ny == ly && nz == lz) || !(isfinite(nx) && isfinite(ny) && isfinite(nz))) return false;
    lx = nx;
    ly = ny;
    lz = nz;
    qx = nx;
    qy = ny;
    qz = nz;
    set_thr(qx, qy, qz);
    return true;
  }

  __device__ bool start(long long idx, double &qx, double &qy, double &qz) {
    if constexpr (MULTI) {
      job = job_of(L.jobs, L.njobs, idx);
      jb = &L.jobs[job];
      fp = P::job_params(L, job);
      kd = P::kind(fp);
    }
    const unsigned long long local = (unsigned long long)(idx - jb->first);
    int x, y;
    if (L.layout == 1) {
      const unsigned long long tile = local >> 5;
      const int w = int(local & 31);
      const unsigned long long ty = fdiv(tile, jb->div_tx);
      x = int(tile - ty * (unsigned long long)jb->tiles_x) * 8 + (w & 7);
      y = int(ty) * 4 + (w >> 3);
    } else {
      const unsigned long long yy = fdiv(local, jb->div_w);
      x = int(local - yy * (unsigned long long)jb->width);
      y = int(yy);
    }
    if (x >= jb->width || y >= jb->rows) return false;  // padding of the last tile row/column
    y += jb->row0;
    ray = unsigned(y) * unsigned(jb->width) + unsigned(x);
    pix = jb->pixel_offset + (long long)ray;
    // camera ray (render_worker.cpp:155-163, 247, 326-327)
    const double ix = (1.0 / double(jb->width) * double(x) + -0.5) * jb->aspect;
    const double iy = jb->legacy_y ? 1.0 / double(jb->height) * double(y) + -0.5
                                   : -1.0 / double(jb->height) * double(y) + 0.5;
    double vx = ix * jb->fov, vy = 1.0, vz = iy * jb->fov;
    if (jb->persp != MBR_PROJECTION_THREE_POINT) {
      if (hemisphere_cut(jb->persp, jb->fov, ix, iy)) {
        last_iters = 0;
        write_miss(true);
        return false;
      }
      const D3 v = projection_dir(jb->persp, jb->fov, ix, iy);
      vx = v.x;
      vy = v.y;
      vz = v.z;
    }
    double n = 1.0 / sqrt(vx * vx + vy * vy + vz * vz);
    vx *= n;
    vy *= n;
    vz *= n;
    if (!jb->mrot_zero) {
      const double *m = jb->mrot;
      const double rx = m[0] * vx + m[1] * vy + m[2] * vz;
      const double ry = m[3] * vx + m[4] * vy + m[5] * vz;
      const double rz = m[6] * vx + m[7] * vy + m[8] * vz;
      vx = rx;
      vy = ry;
      vz = rz;
    }
    n = 1.0 / sqrt(vx * vx + vy * vy + vz * vz);
    dx = vx * n;
    dy = vy * n;
    dz = vz * n;
    dir_len = sqrt(dx * dx + dy * dy + dz * dz);
    ox = jb->cam[0];
    oy = jb->cam[1];
    oz = jb->cam[2];
    c0 = D(jb->c0);
    t = 0.0;
    stp = 0.0;
    phase = 0;
    sub = 0;
    count = 0;
    last_iters = 0;
    thr = D(0);
    lx = ly = lz = 1e30;
    if (fr.jitter) pm = pm_for_ray(ray, fr.seed).s;
    if (!advance(qx, qy, qz)) {  // a camera that is not finite: stuck at once
      write_hit();
      return false;
    }
    return true;
  }

  // cut: a fish-eye-cut pixel, not traced and black
  __device__ void write_miss(bool cut = false) {
    float rgb[3] = {fr.background[0], fr.background[1], fr.background[2]};
    if (cut) rgb[0] = rgb[1] = rgb[2] = 0.0f;
    if (out.depth) out.depth[pix] = 1e20;
    if (out.iters) out.iters[pix] = last_iters;
    if (out.hit) out.hit[pix] = 0;
    if (out.normal) {
      out.normal[3 * pix + 0] = 0.f;
      out.normal[3 * pix + 1] = 0.f;
      out.normal[3 * pix + 2] = 0.f;
    }
    if (out.shade) out.shade[pix] = 0.f;
    if (out.ao) out.ao[pix] = 1.0f;
    if (out.rgb) {
      out.rgb[3 * pix + 0] = rgb[0];
      out.rgb[3 * pix + 1] = rgb[1];
      out.rgb[3 * pix + 2] = rgb[2];
    }
    if (out.rgb8) to_rgb8(fr, rgb, &out.rgb8[3 * pix]);
  }

  __device__ void write_hit() {
    const unsigned long long h = atomicAdd(&L.ctr->hits, 1ull);
    HitRec &r = L.hits[h];
    r.px = fma(dx, t, ox);
    r.py = fma(dy, t, oy);
    r.pz = fma(dz, t, oz);
    r.depth = t;
    r.pix = pix;
    r.thr = double(thr);
    r.iters = last_iters;
    r.nx = 1.f;
    r.ny = 0.f;
    r.nz = 0.f;
    r.shade = 0.f;
    r.shadow = 1.f;
    r.ao_q = 0ull;
    r.job = MULTI ? job : 0;
    r.ray = ray;
  }

  // reference binary search step (render_worker.cpp:854-912)
  __device__ bool binary_check(double &qx, double &qy, double &qz) {
    if (sub >= fr.binary_steps || (dist_prev < thr && dist_prev > thr * search_limit)) {
      write_hit();
      return false;
    }
    if (dist_prev > thr) t += stp;
    else if (dist_prev < thr * search_limit) t -= stp;
    point(qx, qy, qz);
    return true;
  }

  __device__ bool step(D d, int iters, double &qx, double &qy, double &qz) {
    last_iters = iters;
    if (phase == 1) {
      binary_de++;
      dist_prev = d;
      stp *= 0.5;
      sub++;
      return binary_check(qx, qy, qz);
    }
    count++;
    if (d < thr) {
      stp *= 0.5;
      sub = 0;
      dist_prev = d;
      phase = 1;
      return binary_check(qx, qy, qz);
    }
    double jit = 1.0;
    if (fr.jitter) {
      ParkMiller p;
      p.s = pm;
      jit = 1.0 - p.random(1000) / 10000.0;
      pm = p.s;
    }
    if (P::kWide) {
      stp = (double(d) - 0.5 * double(thr)) * fr.de_factor * jit;
      stp = step_limit(fr, stp, double(thr));
      t += stp / dir_len;
    } else {
      stp = double((float(d) - 0.5f * float(thr)) * float(fr.de_factor)) * jit;
      if (fr.adv_quality) stp = step_limit(fr, stp, double(thr));
      else if (stp > 3.0) stp = 3.0;
      t += stp;
    }
    if (t > fr.view_distance_max || count >= fr.max_steps) {
      write_miss();
      return false;
    }
    if (!advance(qx, qy, qz)) {  // stuck: a hit where it stands, without refinement
      write_hit();
      return false;
    }
    return true;
  }
};

template <int FK, bool MULTI, class P>
__global__ void __launch_bounds__(256) primary_kernel(const __grid_constant__ DevFrame fr,
                                                      const __grid_constant__ typename P::Params fp0,
                                                      const __grid_constant__ WJob job0,
                                                      const __grid_constant__ Launch L, DevOutputs out) {
  if (gated_off(L)) return;
  PrimaryStage<MULTI, P> S{fr, L, out, &job0, fp0, P::kind(fp0), 0};
  S.search_limit = typename P::D(1.0 - 0.001 * fr.detail_level);
  S.binary_de = 0;
  unsigned int my_de = 0;
  unsigned long long my_iters = 0;
  run_stage<FK, P>(S, fp0, &L.ctr->pixels_next, L.total, L.refill_k, &my_de, &my_iters);
  flush_counts(out, my_de, my_iters, K_MARCH, my_de - S.binary_de, K_BINARY, S.binary_de);
}

// ============================================================================
// Stage N: normals + Lambert term, one task per hit.
// ============================================================================
template <bool MULTI, class P>
struct NormalStage {
  typedef double Real;
  static constexpr bool kMulti = MULTI;
  typedef typename P::D D;
  const DevFrame &fr;
  const Launch &L;
  typename P::Params fp;
  int kd;
  HitRec *r;
  double ox, oy, oz, delta;
  D thr, nx, ny, nz;
  int sub;

  __device__ const typename P::Params &params() const { return fp; }
  __device__ int kind() const { return kd; }
  __device__ D detail() const { return thr; }

  __device__ void point(double &qx, double &qy, double &qz) {
    const double dd = (sub & 1) ? -delta : delta;
    const int axis = sub >> 1;
    qx = ox + (axis == 0 ? dd : 0.0);
    qy = oy + (axis == 1 ? dd : 0.0);
    qz = oz + (axis == 2 ? dd : 0.0);
  }

  __device__ bool start(long long idx, double &qx, double &qy, double &qz) {
    r = &L.hits[idx];
    if constexpr (MULTI) {
      fp = P::job_params(L, r->job);
      kd = P::kind(fp);
    }
    ox = r->px;
    oy = r->py;
    oz = r->pz;
    thr = D(r->thr);
    delta = r->thr * fr.smoothness;
    sub = 0;
    nx = ny = nz = D(0);
    point(qx, qy, qz);
    return true;
  }

  __device__ bool step(D d, int, double &qx, double &qy, double &qz) {
    const bool neg = (sub & 1) != 0;
    const int axis = sub >> 1;
    D &comp = (axis == 0) ? nx : ((axis == 1) ? ny : nz);
    comp = neg ? comp - d : d;
    sub++;
    if (sub < 6) {
      point(qx, qy, qz);
      return true;
    }
    // CalculateNormals tail (shader_calculate_normals.cpp:111-123)
    float fx, fy, fz;
    float s = 0.f;
    if (P::kWide) {
      double ux = double(nx), uy = double(ny), uz = double(nz);
      if (fabs(ux) < 1e-50 && fabs(uy) < 1e-50 && fabs(uz) < 1e-50) {
        ux = 1.0;
        uy = uz = 0.0;
      } else {
        const double inv = 1.0 / sqrt(ux * ux + uy * uy + uz * uz);
        ux *= inv;
        uy *= inv;
        uz *= inv;
      }
      if (!(isfinite(ux) && isfinite(uy) && isfinite(uz))) {
        ux = 1.0;
        uy = uz = 0.0;
      }
      fx = float(ux);
      fy = float(uy);
      fz = float(uz);
      if (fr.shading_enable) s = float(ux * fr.light[0] + uy * fr.light[1] + uz * fr.light[2]);
    } else {
      fx = float(nx);
      fy = float(ny);
      fz = float(nz);
      if (fabsf(fx) < 1e-30f && fabsf(fy) < 1e-30f && fabsf(fz) < 1e-30f) {
        fx = 1.f;
        fy = fz = 0.f;
      } else {
        const float inv = rsqrtf(fx * fx + fy * fy + fz * fz);
        fx *= inv;
        fy *= inv;
        fz *= inv;
      }
      if (!(isfinite(fx) && isfinite(fy) && isfinite(fz))) {
        fx = 1.f;
        fy = fz = 0.f;
      }
      if (fr.shading_enable) s = fx * float(fr.light[0]) + fy * float(fr.light[1]) + fz * float(fr.light[2]);
    }
    r->nx = fx;
    r->ny = fy;
    r->nz = fz;
    // LightShading, directional light (shader_light_shading.cpp:61-72)
    if (fr.shading_enable) {
      if (s < 0) s = 0;
      s = 1.0f - fr.material_shading + s * fr.material_shading;
      s = s * fr.light_intensity;
      if (s > 500.0f) s = 500.0f;
    }
    r->shade = s;
    return false;
  }
};

template <int FK, bool MULTI, class P>
__global__ void __launch_bounds__(256) normal_kernel(const __grid_constant__ DevFrame fr,
                                                     const __grid_constant__ typename P::Params fp0,
                                                     const __grid_constant__ Launch L, DevOutputs out) {
  if (gated_off(L)) return;
  NormalStage<MULTI, P> S{fr, L, fp0, P::kind(fp0)};
  unsigned int my_de = 0;
  unsigned long long my_iters = 0;
  const long long total = (long long)L.ctr->hits;
  run_stage<FK, P>(S, fp0, &L.ctr->normals_next, total, L.refill_k, &my_de, &my_iters);
  const int slot = L.normal_slot ? L.normal_slot : K_NORMAL;
  flush_counts(out, my_de, my_iters, slot, my_de, slot, 0);
}

// ============================================================================
// Stage S: shadow march and AO marches, (shadow_tasks + ao_rays) tasks per hit.
// ============================================================================
// PCG32 jump-ahead by `delta` steps: Brown, "Random Number Generation with
// Arbitrary Strides" (Trans. Am. Nucl. Soc. 71, 1994), as in pcg32_advance_r.
__device__ __forceinline__ unsigned long long pcg_advance(unsigned long long state, unsigned long long inc,
                                                          unsigned long long delta) {
  unsigned long long cur_mult = 6364136223846793005ull, cur_plus = inc;
  unsigned long long acc_mult = 1ull, acc_plus = 0ull;
  while (delta > 0) {
    if (delta & 1) {
      acc_mult *= cur_mult;
      acc_plus = acc_plus * cur_mult + cur_plus;
    }
    cur_plus = (cur_mult + 1ull) * cur_plus;
    cur_mult *= cur_mult;
    delta >>= 1;
  }
  return acc_mult * state + acc_plus;
}

// The secondary marches run in the policy's precision: FP32 from the FP64
// hit point rounded once (no FP64 conversions in the loop), or FP64 from the
// hit point itself.  Their hit test uses the float-rounded distThresh, as the
// reference's shaders do.
// The march length of a penetrating directional light's shadow: delta /
// resolution at the hit, i.e. |camera - p| * fov (light.cpp:277-290), with
// the camera of the hit's own job
template <bool MULTI>
__device__ __forceinline__ double shadow_distance(const DevFrame &fr, const Launch &L, const HitRec &r) {
  const double *cam = MULTI ? L.jobs[r.job].cam : fr.camera;
  const double res = MULTI ? L.jobs[r.job].resolution : fr.resolution;
  const double fov = MULTI ? L.jobs[r.job].fov : fr.fov;
  const int persp = MULTI ? L.jobs[r.job].persp : fr.persp;
  const double ax = cam[0] - r.px, ay = cam[1] - r.py, az = cam[2] - r.pz;
  double delta = sqrt(ax * ax + ay * ay + az * az) * res * fov;  // CalcDelta
  if (persp == MBR_PROJECTION_EQUIRECTANGULAR) delta *= 0.5;
  return delta / res;
}

// FAST: the AO task is the fast AO (a separate instantiation, so the march
// kernels carry none of its code).
template <bool MULTI, class P, bool FAST>
struct ShadeStage {
  typedef typename P::D Real;
  static constexpr bool kMulti = MULTI;
  typedef typename P::D D;
  const DevFrame &fr;
  const Launch &L;
  typename P::Params fp;
  int kd;
  HitRec *r;
  D ox, oy, oz, t;
  D dx, dy, dz, end, vdm, dfac;
  // soft shadow: the largest 1 - angle / range so far (shader_aux_shadow.cpp:142-151);
  // fast AO: the previous (clamped) distance sample
  D maxsoft;
  float thr;
  int count, mode;  // mode 0 shadow, 1 AO march, 2 fast AO (end: its float sum)
  unsigned int shadow_de;
  unsigned int trips;  // AO marches that reached max_raymarching_steps (watchdog)

  __device__ const typename P::Params &params() const { return fp; }
  __device__ int kind() const { return kd; }
  __device__ D detail() const { return D(thr); }

  __device__ void point(D &qx, D &qy, D &qz) {
    qx = fmadd(dx, t, ox);
    qy = fmadd(dy, t, oy);
    qz = fmadd(dz, t, oz);
  }

  __device__ bool start(long long idx, D &qx, D &qy, D &qz) {
    // both start records are loaded before the first is tested: the origin's
    // address depends on the task index only, so the two loads overlap
    const long long h = (long long)fdiv((unsigned long long)idx, L.div_per);
    const float4 dv = L.sdir[idx];
    float4 o = make_float4(0.f, 0.f, 0.f, 0.f);
    if (!P::kWide) o = L.sorg[h];
    if (dv.w == 0.0f) return false;  // resolved by the direction kernel
    r = &L.hits[h];
    if constexpr (MULTI) {
      fp = P::job_params(L, r->job);
      kd = P::kind(fp);
    }
    if (P::kWide) {
      ox = D(r->px);
      oy = D(r->py);
      oz = D(r->pz);
      thr = float(r->thr);
      t = D(r->thr);
    } else {
      ox = D(o.x);
      oy = D(o.y);
      oz = D(o.z);
      thr = o.w;
      t = D(thr);
    }
    dx = D(dv.x);
    dy = D(dv.y);
    dz = D(dv.z);
    mode = dv.w < 0.0f ? 0 : (FAST ? 2 : 1);
    end = mode == 1 ? D(dv.w) : vdm;
    if (!mode && fr.penetrating) end = D(shadow_distance<MULTI>(fr, L, *r));
    maxsoft = D(0);
    if (FAST && mode == 2) {  // first sample at 1 * distThresh along the normal
      end = D(0);
      maxsoft = D(1e20);
    }
    count = 0;
    point(qx, qy, qz);
    return true;
  }

  __device__ bool step(D d, int, D &qx, D &qy, D &qz) {
    count++;
    if (mode == 0) {
      shadow_de++;
      const bool soft = fr.soft_range > 0.0;
      bool outside = false;  // a soft shadow ignores samples outside the limit box (shader_aux_shadow.cpp:130-147)
      if constexpr (P::kHyb) {
        const DevScene &sc = *fp.sc;
        if (soft && sc.limits) {
          D qx, qy, qz;
          point(qx, qy, qz);
          outside = qx < sc.flim_min[0] || qx > sc.flim_max[0] || qy < sc.flim_min[1] || qy > sc.flim_max[1] ||
                    qz < sc.flim_min[2] || qz > sc.flim_max[2];
        }
      }
      if (soft && !outside) {
        D angle = (d - D(thr)) / t;
        if (angle < D(0)) angle = D(0);
        if (d < D(thr)) angle = D(0);
        D sft = D(1) - angle / D(fr.soft_range);
        if (fr.penetrating) sft = sft * ((end - t) / end);
        if (sft < D(0)) sft = D(0);
        if (sft > maxsoft) maxsoft = sft;
      }
      if (d < D(thr)) {
        D v = D(0);
        if (fr.penetrating) {
          v = D(1) - (end - t) / end;
          if (v < D(0)) v = D(0);
        }
        r->shadow = float(soft ? D(1) - maxsoft : v);
        return false;
      }
      if (P::kWide) t += fmax(fmin(double(d), 1e6) * double(dfac), 1e-15);
      else t += fmaxf(fminf(float(d), 1e6f) * float(dfac), 1e-15f);
      if (count > fr.max_steps || t >= end) {
        r->shadow = soft ? float(D(1) - maxsoft) : 1.f;
        return false;
      }
    } else if (FAST && mode == 2) {
      // FastAmbientOcclusion (shader_fast_ambient_occlusion.cpp:40-65): sample
      // i = count at scan t = i^2 distThresh; the sum is kept in float
      D dist = d;
      if (dist > maxsoft * D(2)) dist = maxsoft * D(2);
      maxsoft = dist;
      const D delta = P::kWide ? D(r->thr) : D(thr);
      if (P::kWide)
        end = D(float(double(end) + ldexp(1.0, -count) * (double(t) - fr.ao_fast_tune * double(dist)) / double(delta)));
      else
        end = D(float(end) + ldexpf(1.0f, -count) * (float(t) - float(fr.ao_fast_tune) * float(dist)) / float(delta));
      const int i = count + 1;
      if (i >= fr.ao_quality * fr.ao_quality) {
        float ao = 1.0f - 0.2f * float(end);
        if (ao < 0.0f) ao = 0.0f;
        r->ao_q = (unsigned long long)__float_as_uint(ao);
        return false;
      }
      t = D(i * i) * delta;
    } else {
      if (d < D(thr)) {
        if (P::kWide) {
          const double s = 1.0 - (double(end) - double(t)) / double(end);
          ao_add(r, fmax(s, 0.0));
        } else {
          const float s = 1.0f - __fdividef(float(end) - float(t), float(end));
          ao_add(r, double(fmaxf(s, 0.0f)));
        }
        return false;
      }
      t = fmadd(D(2), d, t);
      if (t >= end || count >= fr.max_steps) {
        if (!(t >= end)) trips++;  // the cap ended it: a watchdog trip
        ao_add(r, 1.0);
        return false;
      }
    }
    point(qx, qy, qz);
    return true;
  }
};

// Stage D: the start records of stage S, one thread per task.  AO direction
// k of a hit: draws 2k, 2k+1 of PCG32(state ao_seed, stream pixel) mapped to
// a cosine-weighted direction about the normal; task 0 (when the shadow
// march runs) points at the light, or is resolved here when the surface faces
// away (LightShading, shade <= 0.001) or no room is left to march.
template <bool MULTI>
__global__ void __launch_bounds__(256) direction_kernel(const __grid_constant__ DevFrame fr,
                                                        const __grid_constant__ Launch L) {
  if (gated_off(L)) return;
  const long long nh = (long long)L.ctr->hits;
  const int per = L.shadow_tasks + L.ao_rays;
  const long long n = nh * per;
  const float vdm = float(fr.view_distance_max);
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < n;
       idx += (long long)gridDim.x * blockDim.x) {
    const long long h = (long long)fdiv((unsigned long long)idx, L.div_per);
    const int k = int(idx - h * per);
    HitRec &r = L.hits[h];
    const float thr = float(r.thr);
    if (k == 0) L.sorg[h] = make_float4(float(r.px), float(r.py), float(r.pz), thr);
    float4 dv;
    if (k < L.shadow_tasks) {
      if (!(r.shade > 0.001f)) {
        r.shadow = 0.f;
        dv = make_float4(0.f, 0.f, 0.f, 0.f);
      } else if (!(thr < (fr.penetrating ? float(shadow_distance<MULTI>(fr, L, r)) : vdm))) {
        r.shadow = 1.f;
        dv = make_float4(0.f, 0.f, 0.f, 0.f);
      } else {
        dv = make_float4(float(fr.light[0]), float(fr.light[1]), float(fr.light[2]), -1.0f);
      }
    } else if (L.ao_fast) {
      dv = make_float4(r.nx, r.ny, r.nz, 1.0f);  // fast AO: samples along the normal
    } else {
      const int a = k - L.shadow_tasks;
      Pcg32 g = pcg_init(fr.ao_seed, (unsigned long long)r.ray);
      g.state = pcg_advance(g.state, g.inc, 2ull * (unsigned long long)a);
      const float u1 = float(g.uniform()), u2 = float(g.uniform());
      const float nx = r.nx, ny = r.ny, nz = r.nz;
      const float rr = sqrtf(u1);
      float sp, cp;
      __sincosf(6.28318530717958647692f * u2, &sp, &cp);
      const float lx = rr * cp, ly = rr * sp, lz = sqrtf(fmaxf(0.0f, 1.0f - u1));
      const float sg = nz >= 0.0f ? 1.0f : -1.0f;
      const float aa = -1.0f / (sg + nz);
      const float b = nx * ny * aa;
      const float end = float(r.depth) * (MULTI ? L.jobs[r.job].fovf : float(fr.fov));
      if (!(thr < end)) {
        ao_add(&r, 1.0);  // no room to march: unoccluded
        dv = make_float4(0.f, 0.f, 0.f, 0.f);
      } else {
        dv = make_float4(fmaf(1.0f + sg * nx * nx * aa, lx, fmaf(b, ly, nx * lz)),
                         fmaf(sg * b, lx, fmaf(sg + ny * ny * aa, ly, ny * lz)),
                         fmaf(-sg * nx, lx, fmaf(-ny, ly, nz * lz)), end);
      }
    }
    L.sdir[idx] = dv;
  }
}

template <int FK, bool MULTI, class P, bool FAST>
__device__ __forceinline__ void shade_body(const DevFrame &fr, const typename P::Params &fp0, const Launch &L,
                                           DevOutputs &out) {
  if (gated_off(L)) return;
  ShadeStage<MULTI, P, FAST> S{fr, L, fp0, P::kind(fp0)};
  S.shadow_de = 0;
  S.trips = 0;
  S.vdm = typename P::D(fr.view_distance_max);
  S.dfac = typename P::D(fr.de_factor);
  unsigned int my_de = 0;
  unsigned long long my_iters = 0;
  const long long total = (long long)L.ctr->hits * (long long)(L.shadow_tasks + L.ao_rays);
  run_stage<FK, P>(S, fp0, &L.ctr->shade_next, total, L.refill_k, &my_de, &my_iters);
  flush_counts(out, my_de, my_iters, K_AO, my_de - S.shadow_de, K_SHADOW, S.shadow_de);
  const unsigned int trips = __reduce_add_sync(0xffffffffu, S.trips);
  if ((threadIdx.x & 31) == 0 && trips) {
    if (out.stats) atomicAdd(reinterpret_cast<unsigned long long *>(out.stats) + K_WATCHDOG, (unsigned long long)trips);
    if (out.status) atomicOr(out.status, int(STATUS_AO_MARCH_CAP));
  }
}

template <int FK, bool MULTI, class P>
__global__ void __launch_bounds__(256) shade_kernel(const __grid_constant__ DevFrame fr,
                                                    const __grid_constant__ typename P::Params fp0,
                                                    const __grid_constant__ Launch L, DevOutputs out) {
  shade_body<FK, MULTI, P, false>(fr, fp0, L, out);
}

// Stage S when the AO is the fast AO.
template <int FK, bool MULTI, class P>
__global__ void __launch_bounds__(256) shade_fast_kernel(const __grid_constant__ DevFrame fr,
                                                         const __grid_constant__ typename P::Params fp0,
                                                         const __grid_constant__ Launch L, DevOutputs out) {
  shade_body<FK, MULTI, P, true>(fr, fp0, L, out);
}

// ============================================================================
// Stage F: colour and outputs of every hit.
// ============================================================================
__global__ void __launch_bounds__(256) finish_kernel(const __grid_constant__ DevFrame fr,
                                                     const __grid_constant__ Launch L, DevOutputs out) {
  if (gated_off(L)) return;
  const long long nh = (long long)L.ctr->hits;
  for (long long h = (long long)blockIdx.x * blockDim.x + threadIdx.x; h < nh; h += (long long)gridDim.x * blockDim.x) {
    const HitRec &r = L.hits[h];
    const long long pix = r.pix;
    const float shade = r.shade * r.shadow;
    const float ao = L.ao_fast        ? __uint_as_float((unsigned int)r.ao_q)
                     : (L.ao_rays > 0) ? float(double(r.ao_q) * (1.0 / 4294967296.0) / double(L.ao_rays))
                                       : 1.0f;
    const float col = fr.albedo * (shade + fr.ambient * ao);
    float rgb[3] = {col, col, col};
    if (out.depth) out.depth[pix] = r.depth;
    if (out.iters) out.iters[pix] = r.iters;
    if (out.hit) out.hit[pix] = 1;
    const bool nrm = fr.shading_enable || L.ao_rays > 0 || L.want_normal;
    if (out.normal) {
      out.normal[3 * pix + 0] = nrm ? r.nx : 0.f;
      out.normal[3 * pix + 1] = nrm ? r.ny : 0.f;
      out.normal[3 * pix + 2] = nrm ? r.nz : 0.f;
    }
    if (out.shade) out.shade[pix] = shade;
    if (out.ao) out.ao[pix] = ao;
    if (out.rgb) {
      out.rgb[3 * pix + 0] = rgb[0];
      out.rgb[3 * pix + 1] = rgb[1];
      out.rgb[3 * pix + 2] = rgb[2];
    }
    if (out.rgb8) to_rgb8(fr, rgb, &out.rgb8[3 * pix]);
  }
}

// Counts pixels (misses + hits) once per launch, from the stage-P queue size.
__global__ void pixel_count_kernel(const __grid_constant__ Launch L, DevOutputs out, long long pixels) {
  if (gated_off(L)) return;
  if (threadIdx.x == 0 && out.stats) atomicAdd(reinterpret_cast<unsigned long long *>(out.stats) + K_PIXELS,
                                               (unsigned long long)pixels);
}

// ============================================================================
// Precision policy
// ============================================================================
// 1 when the smallest hit threshold of a view, bounded below by
// DE(camera) * c0 (c0: threshold per unit distance), or the constant
// threshold, is below kWideRatio FP32 units of the camera coordinates.  The
// bound passes through the threshold's tail (equirectangular halving,
// advanced-quality clamps) as every threshold of the view does.
__device__ __forceinline__ int wide_needed(const DevScene &sc, const DevFrame &fr, const double cam[3], double c0,
                                           int persp) {
  double thr_min = fr.de_thresh;
  if (!fr.constant_de_threshold) {
    int it;
    const double d0 = calc_distance<double, F_EXT, false>(sc, cam[0], cam[1], cam[2], 0.0, false, &it);
    thr_min = d0 * c0;
  }
  thr_min = thresh_tail(fr, persp, thr_min);
  const double scale = fmax(fmax(fabs(cam[0]), fabs(cam[1])), fmax(fabs(cam[2]), 1.0));
  return (thr_min < kWideRatio * scale * 0x1p-24) ? 1 : 0;
}

__global__ void policy_kernel(const __grid_constant__ DevScene sc, const __grid_constant__ DevFrame fr, int *gate) {
  if (blockIdx.x == 0 && threadIdx.x == 0)
    *gate = wide_needed(sc, fr, fr.camera, fr.resolution * fr.fov / fr.detail_level, fr.persp);
}

__global__ void batch_policy_kernel(const DevScene *scenes, const int *scene_of, const WJob *jobs, int n,
                                    const __grid_constant__ DevFrame fr, int *flags) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n)
    flags[i] = wide_needed(scenes[scene_of[i]], fr, jobs[i].cam, jobs[i].resolution * jobs[i].fov / jobs[i].detail,
                           jobs[i].persp);
}

// ============================================================================
// GI frames (single-frame launches).  Monte Carlo paths of GlobalIlumination
// (src/shader_global_illumination.cpp:41-209) with MonteCarloDOF
// (src/render_worker.cpp:1832-1862), as the plain kernel's gi_path restates
// them, split into stages like the frame pipeline:
//   stage GP  one task per path (pixel, sample), pixel-major: the jittered
//             thin-lens primary ray, the reference march and binary search;
//             a hit appends the path's first vertex to the level-0 list
//   per level b = 0 .. bounces:
//     stage N   the six normal samples of every vertex of level b
//     stage GV  per vertex: the hard sun-shadow march when the surface faces
//               the sun, its radiance term, then (b < bounces) the cosine
//               bounce marched with the GI step rule; a hit appends the next
//               vertex to the level-b+1 list, a miss adds the sky
//   stage GF  per pixel: the path radiances summed in sample order.
// Random numbers come from the same PCG32 stream per (pixel, sample) and the
// same Park-Miller jitter stream as the plain kernel's: the bounce of level b
// takes draws 4 + 2b and 5 + 2b, reached by jump-ahead.  A path's radiance
// terms are added in the plain kernel's order by one thread at a time.
// ============================================================================
enum { G_MARCH = 0, G_BINARY, G_SHADOW, G_BOUNCE };

// distThresh at q (render_worker.cpp:653-679), from the camera position
__device__ __forceinline__ double gi_thresh(const DevFrame &fr, double qx, double qy, double qz) {
  if (fr.constant_de_threshold) return thresh_tail(fr, fr.persp, fr.de_thresh);
  const double ax = fr.camera[0] - qx, ay = fr.camera[1] - qy, az = fr.camera[2] - qz;
  return thresh_tail(fr, fr.persp, sqrt(ax * ax + ay * ay + az * az) * fr.resolution * fr.fov / fr.detail_level);
}

template <class P>
struct GIPrimaryStage {
  typedef double Real;
  typedef typename P::D D;
  static constexpr bool kMulti = false;
  const DevFrame &fr;
  const Launch &L;
  const DevOutputs &out;
  const WJob *jb;
  typename P::Params fp;
  int kd;
  unsigned long long ray;  // RNG stream id: frame pixel * samples + sample
  long long pix;           // output index of the pixel
  long long path;          // path of the launch: pixel of the launch * samples + sample
  int sample, phase, sub, count, last_iters;
  unsigned int pm;
  double ox, oy, oz, dx, dy, dz, t, stp, dir_len, thr;
  double lx, ly, lz;  // previous request point (dead-ray check)
  D dist_prev, search_limit;
  unsigned int n_march, n_binary;

  __device__ const typename P::Params &params() const { return fp; }
  __device__ int kind() const { return kd; }
  __device__ D detail() const { return D(thr); }
  __device__ void ray_point(double &qx, double &qy, double &qz) const {
    qx = ox + dx * t;
    qy = oy + dy * t;
    qz = oz + dz * t;
  }

  __device__ bool start(long long idx, double &qx, double &qy, double &qz) {
    const unsigned long long spp = (unsigned long long)fr.gi_samples;
    path = idx;
    const unsigned long long lpix = fdiv((unsigned long long)idx, L.div_spp);
    sample = int((unsigned long long)idx - lpix * spp);
    const unsigned long long yy = fdiv(lpix, jb->div_w);
    const int x = int(lpix - yy * (unsigned long long)jb->width);
    const int y = int(yy) + jb->row0;
    const unsigned long long pixel = (unsigned long long)y * (unsigned long long)jb->width + (unsigned long long)x;
    pix = jb->pixel_offset + (long long)pixel;
    ray = pixel * spp + (unsigned long long)sample;
    Pcg32 rng = pcg_init(fr.gi_seed, ray);
    const double ujx = rng.uniform(), ujy = rng.uniform(), ulr = rng.uniform(), ula = rng.uniform();
    double ix, iy;
    image_point(fr, double(x), double(y), &ix, &iy);
    if (hemisphere_cut(fr.persp, fr.fov, ix, iy)) {  // not traced: black, no hit
      last_iters = 0;
      if (sample == 0) {
        if (out.depth) out.depth[pix] = 1e20;
        if (out.iters) out.iters[pix] = 0;
        if (out.hit) out.hit[pix] = 0;
      }
      L.path_rad[path] = 0.0;
      return false;
    }
    ix = ix + (ujx - 0.5) / double(fr.width) * fr.aspect;
    iy = iy + (ujy - 0.5) / double(fr.height);
    D3 view = view_vector(fr, ix, iy);
    const D3 cam = camera_of(fr);
    D3 st = cam;
    if (fr.dof_aperture > 0.0) {
      const double randR = fr.dof_aperture * sqrt(ulr);
      const double randAngle = 2.0 * 3.14159265358979323846 * ula;
      double sa, ca;
      sincos(randAngle, &sa, &ca);
      const D3 rv = rotate(fr, D3{randR * sa, 0.0, randR * ca});
      view = d3sub(view, d3mul(rv, 1.0 / fr.dof_focus));
      st = d3add(cam, rv);
    }
    const D3 dir = d3norm(view);
    ox = st.x;
    oy = st.y;
    oz = st.z;
    dx = dir.x;
    dy = dir.y;
    dz = dir.z;
    dir_len = d3len(dir);
    pm = pm_for_ray(ray, fr.seed).s;
    phase = G_MARCH;
    t = 0.0;
    stp = 0.0;
    count = 0;
    sub = 0;
    last_iters = 0;
    thr = 0.0;
    ray_point(qx, qy, qz);
    if (!(isfinite(qx) && isfinite(qy) && isfinite(qz))) {  // stuck at once (render_worker.cpp:747-756)
      hit();
      return false;
    }
    lx = qx;
    ly = qy;
    lz = qz;
    thr = gi_thresh(fr, qx, qy, qz);
    return true;
  }

  __device__ bool miss() {
    if (sample == 0) {
      if (out.depth) out.depth[pix] = 1e20;
      if (out.iters) out.iters[pix] = last_iters;
      if (out.hit) out.hit[pix] = 0;
    }
    L.path_rad[path] = fr.gi_sky;
    return false;
  }

  // the primary ray found the surface at t: the path's first vertex
  __device__ bool hit() {
    if (sample == 0) {
      if (out.depth) out.depth[pix] = t;
      if (out.iters) out.iters[pix] = last_iters;
      if (out.hit) out.hit[pix] = 1;
    }
    L.path_rad[path] = 0.0;
    const unsigned long long h = atomicAdd(&L.ctr->hits, 1ull);
    HitRec &r = L.hits[h];
    ray_point(r.px, r.py, r.pz);
    r.depth = t;
    r.thr = thr;
    r.pix = path;
    r.iters = last_iters;
    r.nx = 1.f;
    r.ny = r.nz = 0.f;
    r.job = 0;
    return false;
  }

  // reference binary search step (render_worker.cpp:854-912)
  __device__ bool binary_check(double &qx, double &qy, double &qz) {
    if (sub >= fr.binary_steps || (double(dist_prev) < thr && double(dist_prev) > thr * double(search_limit)))
      return hit();
    if (double(dist_prev) > thr) t += stp;
    else if (double(dist_prev) < thr * double(search_limit)) t -= stp;
    ray_point(qx, qy, qz);
    thr = gi_thresh(fr, qx, qy, qz);
    return true;
  }

  __device__ bool step(D d, int iters, double &qx, double &qy, double &qz) {
    last_iters = iters;
    if (phase == G_BINARY) {
      n_binary++;
      dist_prev = d;
      stp *= 0.5;
      sub++;
      return binary_check(qx, qy, qz);
    }
    n_march++;
    count++;
    if (double(d) < thr) {
      stp *= 0.5;
      sub = 0;
      dist_prev = d;
      phase = G_BINARY;
      return binary_check(qx, qy, qz);
    }
    double jit = 1.0;
    if (fr.jitter) {
      ParkMiller p;
      p.s = pm;
      jit = 1.0 - p.random(1000) / 10000.0;
      pm = p.s;
    }
    stp = (double(d) - 0.5 * thr) * fr.de_factor * jit;
    stp = step_limit(fr, stp, thr);
    t += stp / dir_len;
    if (t > fr.view_distance_max || count >= fr.max_steps) return miss();
    ray_point(qx, qy, qz);
    if ((qx == lx && qy == ly && qz == lz) || !(isfinite(qx) && isfinite(qy) && isfinite(qz))) return hit();
    lx = qx;
    ly = qy;
    lz = qz;
    thr = gi_thresh(fr, qx, qy, qz);
    return true;
  }
};

template <class P>
struct GIVertexStage {
  typedef double Real;
  typedef typename P::D D;
  static constexpr bool kMulti = false;
  const DevFrame &fr;
  const Launch &L;
  typename P::Params fp;
  int kd;
  long long path;
  int phase, count;
  double tp, vx, vy, vz, vthr, nx, ny, nz, ndl;
  double ox, oy, oz, dx, dy, dz, t, thr;
  unsigned int n_gi;

  __device__ const typename P::Params &params() const { return fp; }
  __device__ int kind() const { return kd; }
  __device__ D detail() const { return D(thr); }
  __device__ void ray_point(double &qx, double &qy, double &qz) const {
    qx = ox + dx * t;
    qy = oy + dy * t;
    qz = oz + dz * t;
  }

  __device__ bool start(long long idx, double &qx, double &qy, double &qz) {
    const HitRec &r = L.hits[idx];
    path = r.pix;
    vx = r.px;
    vy = r.py;
    vz = r.pz;
    vthr = r.thr;
    nx = double(r.nx);
    ny = double(r.ny);
    nz = double(r.nz);
    ndl = nx * fr.light[0] + ny * fr.light[1] + nz * fr.light[2];
    tp = 1.0;
    for (int b = 0; b < L.level; b++) tp *= double(fr.albedo);
    if (!(ndl > 0.0)) return after_shadow(0.0, qx, qy, qz);
    // hard AuxShadow toward the sun from the vertex (shader_aux_shadow.cpp:94-321)
    phase = G_SHADOW;
    t = vthr;
    count = 0;
    thr = vthr;
    if (!(t < fr.view_distance_max)) return after_shadow(1.0, qx, qy, qz);
    ox = vx;
    oy = vy;
    oz = vz;
    dx = fr.light[0];
    dy = fr.light[1];
    dz = fr.light[2];
    ray_point(qx, qy, qz);
    return true;
  }

  __device__ bool after_shadow(double sh, double &qx, double &qy, double &qz) {
    if (ndl > 0.0) L.path_rad[path] += tp * double(fr.albedo) * fr.gi_sun * ndl * sh;
    if (L.level >= fr.gi_bounces) return false;
    tp *= double(fr.albedo);
    // the bounce's two draws of the path's stream
    const unsigned long long spp = (unsigned long long)fr.gi_samples;
    const unsigned long long lpix = fdiv((unsigned long long)path, L.div_spp);
    const unsigned long long sample = (unsigned long long)path - lpix * spp;
    const unsigned long long ray = ((unsigned long long)L.row0 * (unsigned long long)fr.width + lpix) * spp + sample;
    Pcg32 rng = pcg_init(fr.gi_seed, ray);
    rng.state = pcg_advance(rng.state, rng.inc, 4ull + 2ull * (unsigned long long)L.level);
    const double u1 = rng.uniform(), u2 = rng.uniform();
    const D3 d = cosine_dir(D3{nx, ny, nz}, u1, u2);
    dx = d.x;
    dy = d.y;
    dz = d.z;
    ox = vx;
    oy = vy;
    oz = vz;
    phase = G_BOUNCE;
    t = vthr;
    count = 0;
    if (!(t < fr.view_distance_max) || count >= fr.max_steps) {
      L.path_rad[path] += tp * fr.gi_sky;
      return false;
    }
    ray_point(qx, qy, qz);
    thr = gi_thresh(fr, qx, qy, qz);
    return true;
  }

  __device__ bool step(D d, int, double &qx, double &qy, double &qz) {
    n_gi++;
    if (phase == G_SHADOW) {
      if (double(d) < double(float(vthr))) return after_shadow(0.0, qx, qy, qz);
      const double s = fmax(fmin(double(d), 1000000.0) * fr.de_factor, 1e-15);
      count++;
      if (count > fr.max_steps) return after_shadow(1.0, qx, qy, qz);
      t += s;
      if (!(t < fr.view_distance_max)) return after_shadow(1.0, qx, qy, qz);
      ray_point(qx, qy, qz);
      return true;
    }
    // G_BOUNCE: the GI march rule (shader_global_illumination.cpp:75-125)
    if (double(d) < thr) {
      if (t < thr * 2.0) return false;  // the bounce hit its own vertex
      const unsigned long long h = atomicAdd(L.next_hits, 1ull);
      HitRec &r = L.hits_next[h];
      ray_point(r.px, r.py, r.pz);
      r.depth = t;
      r.thr = thr;
      r.pix = path;
      r.iters = 0;
      r.nx = 1.f;
      r.ny = r.nz = 0.f;
      r.job = 0;
      return false;
    }
    count++;
    t += double(d) * fr.de_factor;
    if (!(t < fr.view_distance_max) || count >= fr.max_steps) {
      L.path_rad[path] += tp * fr.gi_sky;
      return false;
    }
    ray_point(qx, qy, qz);
    thr = gi_thresh(fr, qx, qy, qz);
    return true;
  }
};

template <int FK, class P>
__global__ void __launch_bounds__(256) gi_primary_kernel(const __grid_constant__ DevFrame fr,
                                                         const __grid_constant__ typename P::Params fp0,
                                                         const __grid_constant__ WJob job0,
                                                         const __grid_constant__ Launch L, DevOutputs out) {
  if (gated_off(L)) return;
  GIPrimaryStage<P> S{fr, L, out, &job0, fp0, P::kind(fp0)};
  S.search_limit = typename P::D(1.0 - 0.001 * fr.detail_level);
  S.n_march = S.n_binary = 0;
  unsigned int my_de = 0;
  unsigned long long my_iters = 0;
  run_stage<FK, P>(S, fp0, &L.ctr->pixels_next, L.total, L.refill_k, &my_de, &my_iters);
  flush_counts(out, my_de, my_iters, K_MARCH, S.n_march, K_BINARY, S.n_binary);
}

// At most 64 registers (4 blocks of 256 per SM): the stage is latency-bound,
// and twice the resident warps outweigh its few spills (the 4K x 16 spp
// hybrid GI frame: 1.28 -> 1.18 s; at 80 registers 1.21 s).
template <int FK, class P>
__global__ void __launch_bounds__(256, 4) gi_vertex_kernel(const __grid_constant__ DevFrame fr,
                                                           const __grid_constant__ typename P::Params fp0,
                                                           const __grid_constant__ Launch L, DevOutputs out) {
  if (gated_off(L)) return;
  GIVertexStage<P> S{fr, L, fp0, P::kind(fp0)};
  S.n_gi = 0;
  unsigned int my_de = 0;
  unsigned long long my_iters = 0;
  const long long total = (long long)L.ctr->hits;
  run_stage<FK, P>(S, fp0, &L.ctr->shade_next, total, L.refill_k, &my_de, &my_iters);
  flush_counts(out, my_de, my_iters, K_GI, S.n_gi, K_GI, 0);
}

// Stage GF: the mean radiance of every pixel (its paths summed in sample
// order, as the plain kernel sums them), its colour and the outputs the plain
// kernel writes for GI (normal 0, shade 0, AO 1).
__global__ void __launch_bounds__(256) gi_finish_kernel(const __grid_constant__ DevFrame fr,
                                                        const __grid_constant__ WJob job0,
                                                        const __grid_constant__ Launch L, DevOutputs out,
                                                        long long pixels) {
  if (gated_off(L)) return;
  const int spp = fr.gi_samples;
  for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < pixels;
       p += (long long)gridDim.x * blockDim.x) {
    const long long pix = job0.pixel_offset + (long long)job0.row0 * job0.width + p;
    double acc = 0.0;
    for (int s = 0; s < spp; s++) acc += L.path_rad[p * spp + s];
    const float v = float(acc / double(spp));
    float rgb[3] = {v, v, v};
    if (out.normal) {
      out.normal[3 * pix + 0] = 0.f;
      out.normal[3 * pix + 1] = 0.f;
      out.normal[3 * pix + 2] = 0.f;
    }
    if (out.shade) out.shade[pix] = 0.f;
    if (out.ao) out.ao[pix] = 1.0f;
    if (out.rgb) {
      out.rgb[3 * pix + 0] = v;
      out.rgb[3 * pix + 1] = v;
      out.rgb[3 * pix + 2] = v;
    }
    if (out.rgb8) to_rgb8(fr, rgb, &out.rgb8[3 * pix]);
  }
}

// ---- host side -------------------------------------------------------------------
static WJob make_job(const DevFrame &fr, long long first, long long pixel_offset) {
  WJob j;
  std::memset(&j, 0, sizeof(j));
  for (int i = 0; i < 3; i++) j.cam[i] = fr.camera[i];
  for (int i = 0; i < 9; i++) j.mrot[i] = fr.mrot[i];
  j.mrot_zero = fr.mrot_zero;
  j.width = fr.width;
  j.height = fr.height;
  j.tiles_x = (fr.width + 7) / 8;
  j.row0 = fr.row0;
  j.rows = fr.row1 - fr.row0;
  j.first = first;
  j.pixel_offset = pixel_offset;
  j.fov = fr.fov;
  j.persp = fr.persp;
  j.legacy_y = fr.legacy_y;
  j.aspect = fr.aspect;
  j.resolution = fr.resolution;
  j.detail = fr.detail_level;
  // CalcDistThresh and CalcDelta halve both for an equirectangular view (render_worker.cpp:669, 688)
  const double half = fr.persp == MBR_PROJECTION_EQUIRECTANGULAR ? 0.5 : 1.0;
  j.c0 = float(fr.resolution * fr.fov / fr.detail_level * half);
  j.fovf = float(fr.fov * half);
  j.cthr = float(fr.de_thresh * half);
  j.div_w = make_fastdiv(j.width);
  j.div_tx = make_fastdiv(j.tiles_x);
  return j;
}

static long long job_items(const WJob &j, int layout) {
  if (layout == 1) return (long long)j.tiles_x * ((j.rows + 3) / 4) * 32;
  return (long long)j.width * j.rows;
}

static mbr_status check_supported(mbr_ctx *ctx, const DevScene &sc, const DevFrame &fr, bool batch) {
  if (batch && (sc.is_hybrid || sc.generic || fr.gi_samples > 0))
    return set_err(ctx, MBR_EUNSUPPORTED,
                   "wavefront batches: hybrid sequences, formulas without a specialised form and GI render one frame "
                   "at a time");
  if (sc.iter_thresh || sc.interior || sc.has_w)
    return set_err(ctx, MBR_EUNSUPPORTED,
                   "wavefront engine: iteration_threshold_mode, interior_mode and initial_waxis != 0 use the plain engines");
  if (sc.delta_de)
    return set_err(ctx, MBR_EUNSUPPORTED,
                   "wavefront engine: the delta DE offsets points by 1e-5 of the detail size, which FP32 points do "
                   "not resolve; it runs on the plain FP64 engines");
  if (fr.refine != MBR_REFINE_REFERENCE)
    return set_err(ctx, MBR_EUNSUPPORTED, "wavefront engine: root refinement uses the plain engines");
  if (sc.n_nodes > 0)
    return set_err(ctx, MBR_EUNSUPPORTED, "wavefront engine: explicit objects trees use the plain engines");
  for (int k = 0; k < MBR_MAX_FRACTALS; k++)
    if (sc.slot[k].add_bail || keyed_formula_has_state(sc.slot[k].formula))
      return set_err(ctx, MBR_EUNSUPPORTED,
                     "wavefront engine: formulas with a convergence bailout or orbit state (pseudo-Kleinian, "
                     "Abox mod 11, box fold bulb pow 2 V2) use the plain engines");
  if (fr.slow_shading)
    return set_err(ctx, MBR_EUNSUPPORTED, "wavefront engine: slow shading (iteration-count normals) uses the plain "
                                          "engines");
  return MBR_OK;
}

static int sm_count() {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms;
}

// The stage launches of one frame or batch under policy P, in stream order.
template <bool MULTI, class P>
static int launch_pipeline(int fk, const mbr_tuning &tu, cudaStream_t st, const DevFrame &fr,
                           const typename P::Params &fp0, const WJob &j0, const Launch &L0, const DevOutputs &out,
                           long long pixels) {
  Launch L = L0;
  L.div_per = make_fastdiv(std::max(1, L.shadow_tasks + L.ao_rays));
  L.gate_value = P::kWide;
  const int sms = sm_count();
  const int grid = std::max(1, sms * tu.ctas_per_sm);
  const int block = tu.block_size;
  if (P::kHyb) fk = FK_ANY;
  int e = int(cudaMemsetAsync(L.ctr, 0, sizeof(Counters4), st));
  if (e) return e;
  if constexpr (!MULTI) {
    if (fr.gi_samples > 0) {  // GI frame: stage GP, then per level stages N and GV, then GF
      L.div_spp = make_fastdiv(fr.gi_samples);
      L.row0 = fr.row0;
      Counters4 *ctrs = L.ctr;
      HitRec *lists[2] = {L.hits, L.hits_next};
      e = int(cudaMemsetAsync(ctrs, 0, sizeof(Counters4) * size_t(fr.gi_bounces + 2), st));
      if (e) return e;
#define GI_CASES(LAUNCH)         \
  switch (fk) {                  \
    LAUNCH(FK_BOX_SIMPLE)        \
    LAUNCH(FK_BOX)               \
    LAUNCH(FK_BULB)              \
    LAUNCH(FK_MENGER)            \
    LAUNCH(FK_ANY)               \
    default: return int(cudaErrorInvalidValue); \
  }
      {
        Launch Lp = L;
        Lp.ctr = &ctrs[0];
        Lp.hits = lists[0];
#define GP_LAUNCH(K) \
  case K:            \
    if constexpr (!P::kHyb || K == FK_ANY) gi_primary_kernel<K, P><<<grid, block, 0, st>>>(fr, fp0, j0, Lp, out); \
    break;
        GI_CASES(GP_LAUNCH)
#undef GP_LAUNCH
      }
      for (int b = 0; b <= fr.gi_bounces; b++) {
        Launch Lb = L;
        Lb.ctr = &ctrs[b];
        Lb.hits = lists[b & 1];
        Lb.hits_next = lists[(b + 1) & 1];
        Lb.next_hits = &ctrs[b + 1].hits;
        Lb.level = b;
        Lb.normal_slot = K_GI;
#define GV_LAUNCH(K)                                                                                   \
  case K:                                                                                              \
    if constexpr (!P::kHyb || K == FK_ANY) {                                                           \
      normal_kernel<K, false, P><<<grid, block, 0, st>>>(fr, fp0, Lb, out);                             \
      gi_vertex_kernel<K, P><<<grid, block, 0, st>>>(fr, fp0, Lb, out);                                 \
    }                                                                                                  \
    break;
        GI_CASES(GV_LAUNCH)
#undef GV_LAUNCH
      }
#undef GI_CASES
      gi_finish_kernel<<<sms * 4, 256, 0, st>>>(fr, j0, L, out, pixels);
      pixel_count_kernel<<<1, 32, 0, st>>>(L, out, pixels);
      return int(cudaGetLastError());
    }
  }
#define STAGE_LAUNCH(KERNEL, K, ...)                                                    \
  case K:                                                                               \
    if constexpr (!P::kHyb || K == FK_ANY) KERNEL<K, MULTI, P><<<grid, block, 0, st>>>(__VA_ARGS__); \
    break;
#define STAGE(KERNEL, ...)                                                              \
  switch (fk) {                                                                         \
    STAGE_LAUNCH(KERNEL, FK_BOX_SIMPLE, __VA_ARGS__)                                    \
    STAGE_LAUNCH(KERNEL, FK_BOX, __VA_ARGS__)                                           \
    STAGE_LAUNCH(KERNEL, FK_BULB, __VA_ARGS__)                                          \
    STAGE_LAUNCH(KERNEL, FK_MENGER, __VA_ARGS__)                                        \
    STAGE_LAUNCH(KERNEL, FK_ANY, __VA_ARGS__)                                           \
    default: return int(cudaErrorInvalidValue);                                         \
  }
  STAGE(primary_kernel, fr, fp0, j0, L, out)
  const bool need_normal = fr.shading_enable || L.ao_rays > 0 || L.want_normal;
  if (need_normal) { STAGE(normal_kernel, fr, fp0, L, out) }
  if (L.ao_rays > 0 || L.shadow_tasks > 0) {
    direction_kernel<MULTI><<<sms * 8, 256, 0, st>>>(fr, L);
    if (L.ao_fast) {
      STAGE(shade_fast_kernel, fr, fp0, L, out)
    } else {
      STAGE(shade_kernel, fr, fp0, L, out)
    }
  }
#undef STAGE
#undef STAGE_LAUNCH
  finish_kernel<<<sms * 4, 256, 0, st>>>(fr, L, out);
  pixel_count_kernel<<<1, 32, 0, st>>>(L, out, pixels);
  return int(cudaGetLastError());
}

// Scratch of a launch over `pixels` work items with `per` stage-S tasks per
// hit: counters and the policy flag (256 B), hit records, FP32 origins and
// stage-S start records.  A HitRec is 88 bytes, so the hit region is rounded
// up to a multiple of 256 bytes: the float4 records after it then start on a
// 16-byte boundary for every pixel count, odd ones included.
static size_t hit_region_bytes(long long pixels) { return (size_t(pixels) * sizeof(HitRec) + 255) / 256 * 256; }

static size_t scratch_bytes(long long pixels, int per) {
  return 256 + hit_region_bytes(pixels) + size_t(pixels) * sizeof(float4) * (1 + size_t(per));
}

// Byte offsets of the hit records, the FP32 origins and the stage-S records.
static void scratch_offsets(long long pixels, size_t off[3]) {
  off[0] = 256;
  off[1] = 256 + hit_region_bytes(pixels);
  off[2] = off[1] + size_t(pixels) * sizeof(float4);
}

static void scratch_layout(Launch &L, void *base, long long pixels) {
  char *p = static_cast<char *>(base);
  size_t off[3];
  scratch_offsets(pixels, off);
  L.ctr = reinterpret_cast<Counters4 *>(p);
  L.gate = nullptr;
  L.hits = reinterpret_cast<HitRec *>(p + off[0]);
  L.sorg = reinterpret_cast<float4 *>(p + off[1]);
  L.sdir = reinterpret_cast<float4 *>(p + off[2]);
}

static int *scratch_gate(void *base) { return reinterpret_cast<int *>(static_cast<char *>(base) + 128); }

static bool is_wavefront(int engine) {
  return engine == MBR_ENGINE_WAVEFRONT_FP32 || engine == MBR_ENGINE_WAVEFRONT_FP64 ||
         engine == MBR_ENGINE_WAVEFRONT_AUTO;
}

mbr_status render_wavefront(mbr_ctx *ctx, const DevScene &sc, const DevFrame &fr, const DevOutputs &out, int engine,
                            void *stream) {
  if (!is_wavefront(engine)) return set_err(ctx, MBR_EINVAL, "not a wavefront engine: %d", engine);
  mbr_status stt = check_supported(ctx, sc, fr, false);
  if (stt != MBR_OK) return stt;
  // hybrids and formulas without a specialised form iterate in the reference's order (PrecHyb)
  const bool gi = fr.gi_samples > 0, hyb = sc.is_hybrid != 0 || sc.generic != 0;
  if (gi && fr.gi_bounces > 120)
    return set_err(ctx, MBR_EUNSUPPORTED, "wavefront engine: GI with more than 120 bounces uses the plain engines");
  if (hyb && engine == MBR_ENGINE_WAVEFRONT_FP64)
    return set_err(ctx, MBR_EUNSUPPORTED, "wavefront engine: hybrid sequences and formulas other than the Mandelbulb, "
                                          "Mandelbox and Menger sponge iterate in FP32 (MBR_ENGINE_WAVEFRONT_FP32 or "
                                          "_AUTO); in FP64 they use MBR_ENGINE_PLAIN_FP64");
  const mbr_tuning tu = ctx_tuning(ctx);
  const WJob j0 = make_job(fr, 0, out.pixel_offset);
  const long long pixels = (long long)fr.width * (fr.row1 - fr.row0);
  const long long total = gi ? pixels * (long long)fr.gi_samples : job_items(j0, tu.queue_layout);
  const int per = ((fr.shading_enable && fr.shadow_enable) ? 1 : 0) + ao_tasks(fr);
  // scratch: counters, then the GI accumulators or the hit records, then (a
  // hybrid scene) the scene the iteration reads
  // GI: a counter block per bounce level (4 KiB), the auto-engine flag, the
  // path radiances and two vertex lists of one entry per path
  const size_t gi_head = 4096 + 256;
  const size_t main_bytes = gi ? gi_head + size_t(total) * (sizeof(double) + 2 * sizeof(HitRec))
                               : scratch_bytes(total, per);
  const size_t scene_at = (main_bytes + 255) / 256 * 256;
  const size_t bytes = hyb ? scene_at + sizeof(DevScene) : main_bytes;
  unsigned long long *work = nullptr;
  stt = ctx_work(ctx, (bytes + 7) / 8, &work);
  if (stt != MBR_OK) return stt;
  Launch L;
  std::memset(&L, 0, sizeof(L));
  L.jobs = nullptr;
  L.fps = nullptr;
  L.wps = nullptr;
  L.njobs = 1;
  L.total = total;
  if (gi) {
    char *w = reinterpret_cast<char *>(work);
    L.ctr = reinterpret_cast<Counters4 *>(w);
    L.path_rad = reinterpret_cast<double *>(w + gi_head);
    L.hits = reinterpret_cast<HitRec *>(w + gi_head + sizeof(double) * size_t(total));
    L.hits_next = L.hits + total;
  } else {
    scratch_layout(L, work, total);
  }
  L.refill_k = tu.refill_k;
  L.layout = tu.queue_layout;
  L.ao_rays = ao_tasks(fr);
  L.ao_fast = fr.ao_fast;
  L.shadow_tasks = (fr.shading_enable && fr.shadow_enable) ? 1 : 0;
  L.want_normal = fr.want_normal;
  const FastParams fp = load_fast_params(sc);
  const WideParams wp = load_wide_params(sc);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int e = 0;
  if (hyb) {  // FP32 hybrid iteration reading the scene from the scratch
    DevScene *d_sc = reinterpret_cast<DevScene *>(reinterpret_cast<char *>(work) + scene_at);
    e = int(cudaMemcpyAsync(d_sc, &sc, sizeof(DevScene), cudaMemcpyHostToDevice, s));
    if (!e)
      e = scene_extended(sc)
              ? launch_pipeline<false, PrecHybT<true>>(FK_ANY, tu, s, fr, HybParams{d_sc}, j0, L, out, pixels)
              : launch_pipeline<false, PrecHyb>(FK_ANY, tu, s, fr, HybParams{d_sc}, j0, L, out, pixels);
    return cuda_err(ctx, e, "wavefront launch");
  }
  if (engine == MBR_ENGINE_WAVEFRONT_AUTO) {
    int *gate = gi ? reinterpret_cast<int *>(reinterpret_cast<char *>(work) + 4096) : scratch_gate(work);
    L.gate = gate;
    policy_kernel<<<1, 32, 0, s>>>(sc, fr, gate);
    e = int(cudaGetLastError());
  }
  if (!e && engine != MBR_ENGINE_WAVEFRONT_FP64)
    e = launch_pipeline<false, Prec32>(fast_kind(fp), tu, s, fr, fp, j0, L, out, pixels);
  if (!e && engine != MBR_ENGINE_WAVEFRONT_FP32)
    e = launch_pipeline<false, Prec64>(wide_kind(wp), tu, s, fr, wp, j0, L, out, pixels);
  return cuda_err(ctx, e, "wavefront launch");
}

}  // namespace mbr

// ============================================================================
// Batches and the autotuner
// ============================================================================
using namespace mbr;

// One pipeline of a batch: the jobs of one formula kind and one precision.
struct BatchGroup {
  int wide;              // 1: Prec64
  int kind;              // FK_* of its jobs
  int offset, count;     // jobs [offset, offset + count) of the batch's job table
  long long items;       // work items of its pixel queue
  long long pixels;
};

struct mbr_batch {
  mbr_ctx *ctx = nullptr;
  WJob *d_jobs = nullptr;
  FastParams *d_params = nullptr;
  WideParams *d_wide = nullptr;
  void *d_scratch = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  long long total = 0;
  std::vector<BatchGroup> groups;
};

// Precision flag of every job (AUTO): the policy kernel over the job table.
static int batch_policy(const std::vector<DevScene> &dsc, const std::vector<int> &scene_of,
                        const std::vector<WJob> &wj, const DevFrame &fr0, std::vector<int> *flags) {
  const int n = int(wj.size());
  DevScene *d_sc = nullptr;
  int *d_of = nullptr, *d_fl = nullptr;
  WJob *d_wj = nullptr;
  int e = int(cudaMalloc(&d_sc, sizeof(DevScene) * dsc.size()));
  if (!e) e = int(cudaMalloc(&d_of, sizeof(int) * n));
  if (!e) e = int(cudaMalloc(&d_fl, sizeof(int) * n));
  if (!e) e = int(cudaMalloc(&d_wj, sizeof(WJob) * n));
  if (!e) e = int(cudaMemcpy(d_sc, dsc.data(), sizeof(DevScene) * dsc.size(), cudaMemcpyHostToDevice));
  if (!e) e = int(cudaMemcpy(d_of, scene_of.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
  if (!e) e = int(cudaMemcpy(d_wj, wj.data(), sizeof(WJob) * n, cudaMemcpyHostToDevice));
  if (!e) {
    batch_policy_kernel<<<(n + 127) / 128, 128>>>(d_sc, d_of, d_wj, n, fr0, d_fl);
    e = int(cudaGetLastError());
  }
  flags->assign(n, 0);
  if (!e) e = int(cudaMemcpy(flags->data(), d_fl, sizeof(int) * n, cudaMemcpyDeviceToHost));
  cudaFree(d_sc);
  cudaFree(d_of);
  cudaFree(d_fl);
  cudaFree(d_wj);
  return e;
}

extern "C" {

mbr_status mbr_batch_create(mbr_ctx *ctx, const mbr_scene *scenes, int32_t n_scenes, const mbr_job *jobs,
                            int32_t n_jobs, const mbr_render_params *params, const mbr_outputs *outs, int engine,
                            void *stream, mbr_batch **batch) {
  if (!batch) return set_err(ctx, MBR_EINVAL, "null batch pointer");
  *batch = nullptr;
  if (!ctx || !scenes || !jobs || !params || !outs || n_scenes < 1 || n_jobs < 1)
    return set_err(ctx, MBR_EINVAL, "null argument or empty batch");
  if (!is_wavefront(engine)) return set_err(ctx, MBR_EUNSUPPORTED, "batches run on the wavefront engines");
  const mbr_tuning tu = ctx_tuning(ctx);
  std::vector<DevScene> dsc(n_scenes);
  for (int i = 0; i < n_scenes; i++) {
    mbr_status st = build_scene(ctx, scenes[i], &dsc[i]);
    if (st != MBR_OK) return st;
  }
  DevFrame fr0;
  std::vector<WJob> wj(n_jobs);
  std::vector<int> scene_of(n_jobs);
  std::vector<long long> job_pixels(n_jobs);
  for (int i = 0; i < n_jobs; i++) {
    const mbr_job &jb = jobs[i];
    if (jb.scene_index < 0 || jb.scene_index >= n_scenes)
      return set_err(ctx, MBR_EINVAL, "job %d: scene_index %d out of range", i, jb.scene_index);
    if (jb.pixel_offset < 0) return set_err(ctx, MBR_EINVAL, "job %d: negative pixel_offset", i);
    DevFrame fr;
    mbr_status st = build_frame(ctx, jb.camera, *params, &fr, stream);
    if (st != MBR_OK) return st;
    st = check_supported(ctx, dsc[jb.scene_index], fr, true);
    if (st != MBR_OK) return st;
    if (i == 0) fr0 = fr;
    wj[i] = make_job(fr, 0, jb.pixel_offset);
    scene_of[i] = jb.scene_index;
    job_pixels[i] = (long long)fr.width * (fr.row1 - fr.row0);
  }
  fr0.want_normal = outs->normal != nullptr;
  {  // the gamma table was copied on `stream`; the graph may be launched on another
    const int e = int(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
    if (e) return cuda_err(ctx, e, "cudaStreamSynchronize");
  }
  // precision of every job
  std::vector<int> wide(n_jobs, engine == MBR_ENGINE_WAVEFRONT_FP64 ? 1 : 0);
  if (engine == MBR_ENGINE_WAVEFRONT_AUTO) {
    const int e = batch_policy(dsc, scene_of, wj, fr0, &wide);
    if (e) return cuda_err(ctx, e, "batch precision policy");
  }
  // groups of one (precision, formula kind), each a contiguous run of the job table
  std::map<std::pair<int, int>, std::vector<int>> by_group;
  for (int i = 0; i < n_jobs; i++) {
    const DevScene &sc = dsc[scene_of[i]];
    const int kind = wide[i] ? wide_kind(load_wide_params(sc)) : fast_kind(load_fast_params(sc));
    by_group[{wide[i], kind}].push_back(i);
  }
  mbr_batch *b = new mbr_batch();
  b->ctx = ctx;
  std::vector<WJob> tab;
  std::vector<FastParams> fps;
  std::vector<WideParams> wps;
  tab.reserve(n_jobs);
  fps.reserve(n_jobs);
  wps.reserve(n_jobs);
  long long max_items = 0;
  for (const auto &kv : by_group) {
    BatchGroup g;
    g.wide = kv.first.first;
    g.kind = kv.first.second;
    g.offset = int(tab.size());
    g.count = int(kv.second.size());
    g.items = 0;
    g.pixels = 0;
    for (int i : kv.second) {
      WJob j = wj[i];
      j.first = g.items;
      g.items += job_items(j, tu.queue_layout);
      g.pixels += job_pixels[i];
      tab.push_back(j);
      fps.push_back(load_fast_params(dsc[scene_of[i]]));
      wps.push_back(load_wide_params(dsc[scene_of[i]]));
    }
    max_items = std::max(max_items, g.items);
    b->groups.push_back(g);
  }
  b->total = 0;
  for (const BatchGroup &g : b->groups) b->total += g.items;
  auto fail = [&](int e, const char *what) {
    mbr_batch_destroy(b);
    return cuda_err(ctx, e, what);
  };
  int e = int(cudaMalloc(&b->d_jobs, sizeof(WJob) * n_jobs));
  if (e) return fail(e, "cudaMalloc(jobs)");
  e = int(cudaMalloc(&b->d_params, sizeof(FastParams) * n_jobs));
  if (e) return fail(e, "cudaMalloc(params)");
  e = int(cudaMalloc(&b->d_wide, sizeof(WideParams) * n_jobs));
  if (e) return fail(e, "cudaMalloc(wide params)");
  const int per = ((fr0.shading_enable && fr0.shadow_enable) ? 1 : 0) + ao_tasks(fr0);
  e = int(cudaMalloc(&b->d_scratch, scratch_bytes(max_items, per)));
  if (e) return fail(e, "cudaMalloc(scratch)");
  e = int(cudaMemcpy(b->d_jobs, tab.data(), sizeof(WJob) * n_jobs, cudaMemcpyHostToDevice));
  if (e) return fail(e, "cudaMemcpy(jobs)");
  e = int(cudaMemcpy(b->d_params, fps.data(), sizeof(FastParams) * n_jobs, cudaMemcpyHostToDevice));
  if (e) return fail(e, "cudaMemcpy(params)");
  e = int(cudaMemcpy(b->d_wide, wps.data(), sizeof(WideParams) * n_jobs, cudaMemcpyHostToDevice));
  if (e) return fail(e, "cudaMemcpy(wide params)");
  // capture the groups' pipelines of one batch into a graph
  cudaStream_t cs;
  e = int(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
  if (e) return fail(e, "cudaStreamCreate");
  const DevOutputs d = dev_outputs(ctx, *outs);
  e = int(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
  if (!e) {
    int le = 0;
    for (const BatchGroup &g : b->groups) {
      Launch L;
      std::memset(&L, 0, sizeof(L));
      L.jobs = b->d_jobs + g.offset;
      L.fps = b->d_params + g.offset;
      L.wps = b->d_wide + g.offset;
      L.njobs = g.count;
      L.total = g.items;
      scratch_layout(L, b->d_scratch, g.items);
      L.refill_k = tu.refill_k;
      L.layout = tu.queue_layout;
      L.ao_rays = ao_tasks(fr0);
      L.ao_fast = fr0.ao_fast;
      L.shadow_tasks = (fr0.shading_enable && fr0.shadow_enable) ? 1 : 0;
      L.want_normal = fr0.want_normal;
      if (g.wide)
        le = launch_pipeline<true, Prec64>(g.kind, tu, cs, fr0, wps[g.offset], tab[g.offset], L, d, g.pixels);
      else
        le = launch_pipeline<true, Prec32>(g.kind, tu, cs, fr0, fps[g.offset], tab[g.offset], L, d, g.pixels);
      if (le) break;
    }
    cudaGraph_t gr = nullptr;
    e = int(cudaStreamEndCapture(cs, &gr));
    b->graph = gr;
    if (!e) e = le;
  }
  cudaStreamDestroy(cs);
  if (e) return fail(e, "graph capture");
  e = int(cudaGraphInstantiate(&b->exec, b->graph, 0));
  if (e) return fail(e, "cudaGraphInstantiate");
  *batch = b;
  return MBR_OK;
}

mbr_status mbr_batch_launch(mbr_batch *b, void *stream) {
  if (!b) return MBR_EINVAL;
  const int e = int(cudaGraphLaunch(b->exec, static_cast<cudaStream_t>(stream)));
  return cuda_err(b->ctx, e, "cudaGraphLaunch");
}

void mbr_batch_destroy(mbr_batch *b) {
  if (!b) return;
  if (b->exec) cudaGraphExecDestroy(b->exec);
  if (b->graph) cudaGraphDestroy(b->graph);
  if (b->d_jobs) cudaFree(b->d_jobs);
  if (b->d_params) cudaFree(b->d_params);
  if (b->d_wide) cudaFree(b->d_wide);
  if (b->d_scratch) cudaFree(b->d_scratch);
  delete b;
}

mbr_status mbr_choose_precision(mbr_ctx *ctx, const mbr_camera *camera, const mbr_render_params *params,
                                int32_t *fp64) {
  if (!ctx || !camera || !params || !fp64) return set_err(ctx, MBR_EINVAL, "null argument");
  const DevScene *sc = ctx_scene(ctx);
  if (!sc) return set_err(ctx, MBR_EINVAL, "no scene set (call mbr_scene_set first)");
  if (cudaSetDevice(ctx_device(ctx)) != cudaSuccess) return set_err(ctx, MBR_ECUDA, "cudaSetDevice failed");
  DevFrame fr;
  mbr_status st = build_frame(ctx, *camera, *params, &fr, nullptr);
  if (st != MBR_OK) return st;
  int *d_flag = nullptr;
  int e = int(cudaMalloc(&d_flag, sizeof(int)));
  if (e) return cuda_err(ctx, e, "cudaMalloc(flag)");
  policy_kernel<<<1, 32>>>(*sc, fr, d_flag);
  e = int(cudaGetLastError());
  int flag = 0;
  if (!e) e = int(cudaMemcpy(&flag, d_flag, sizeof(int), cudaMemcpyDeviceToHost));
  cudaFree(d_flag);
  if (e) return cuda_err(ctx, e, "precision policy");
  *fp64 = flag;
  return MBR_OK;
}

mbr_status mbr_wavefront_scratch_layout(int64_t pixels, int32_t tasks_per_hit, uint64_t offsets[3],
                                        uint64_t *total_bytes) {
  if (pixels < 0 || tasks_per_hit < 0 || !offsets || !total_bytes) return MBR_EINVAL;
  size_t off[3];
  scratch_offsets(pixels, off);
  for (int i = 0; i < 3; i++) offsets[i] = off[i];
  *total_bytes = scratch_bytes(pixels, tasks_per_hit);
  return MBR_OK;
}

int32_t mbr_batch_groups(const mbr_batch *b, int32_t *wide_jobs) {
  if (!b) return -1;
  int32_t w = 0;
  for (const BatchGroup &g : b->groups)
    if (g.wide) w += g.count;
  if (wide_jobs) *wide_jobs = w;
  return int32_t(b->groups.size());
}

// Times the wavefront pipeline on the given frame over block size x CTAs per
// SM x refill threshold x queue layout and keeps the fastest configuration.
mbr_status mbr_autotune(mbr_ctx *ctx, const mbr_camera *camera, const mbr_render_params *params,
                        const mbr_outputs *out, int engine, void *stream, mbr_tuning *best) {
  if (!ctx || !camera || !params || !out || !best) return set_err(ctx, MBR_EINVAL, "null argument");
  const mbr_tuning saved = ctx_tuning(ctx);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  mbr_tuning bt = saved;
  const int blocks[] = {128, 256};  // __launch_bounds__(256)
  const int ctas[] = {6, 8, 12};
  const int ks[] = {0, 2, 4, 8, 16, 24};
  const int layouts[] = {0, 1};
  mbr_status status = MBR_OK;
  // one timed frame per launch shape, then the four fastest re-timed three
  // times each: the median decides (a single frame can be lucky by several
  // per cent, more than the shapes differ)
  std::vector<std::pair<float, mbr_tuning>> cand;
  auto time_one = [&](const mbr_tuning &t, float *ms) {
    ctx_tuning(ctx) = t;
    mbr_status s2 = mbr_render(ctx, camera, params, out, engine, stream);  // warm-up
    if (s2 != MBR_OK) return s2;
    cudaEventRecord(e0, st);
    s2 = mbr_render(ctx, camera, params, out, engine, stream);
    cudaEventRecord(e1, st);
    if (s2 != MBR_OK) return s2;
    cudaEventSynchronize(e1);
    cudaEventElapsedTime(ms, e0, e1);
    return MBR_OK;
  };
  for (int b : blocks)
    for (int c : ctas) {
      if (b * c > 2048) continue;
      for (int k : ks)
        for (int l : layouts) {
          const mbr_tuning t{b, c, k, l};
          float ms = 0.f;
          status = time_one(t, &ms);
          if (status != MBR_OK) goto done;
          cand.push_back({ms, t});
        }
    }
  std::sort(cand.begin(), cand.end(),
            [](const std::pair<float, mbr_tuning> &a, const std::pair<float, mbr_tuning> &b) { return a.first < b.first; });
  {
    float best_ms = 1e30f;
    for (size_t i = 0; i < cand.size() && i < 4; i++) {
      float m[3];
      for (int r = 0; r < 3; r++) {
        status = time_one(cand[i].second, &m[r]);
        if (status != MBR_OK) goto done;
      }
      std::sort(m, m + 3);
      if (m[1] < best_ms) {
        best_ms = m[1];
        bt = cand[i].second;
      }
    }
  }
done:
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  ctx_tuning(ctx) = (status == MBR_OK) ? bt : saved;
  *best = ctx_tuning(ctx);
  return status;
}

}  // extern "C"

// ============================================================================
// Allocation-free rendering
//
// For callers that cannot allocate device memory: a host application whose
// device memory is owned by its own allocator or memory pool (which must not
// be bypassed), or a process running under a hard memory cap, where a
// cudaMalloc in the middle of a frame could fail or synchronise the device.
// The wavefront pipeline's scratch (hit records, stage-S start records,
// launch counters, the gamma table and the status word) lives in one
// file-scope device array, part of this library's device image: every GPU
// that loads the library holds it until the process exits.
// ============================================================================
namespace {

static __device__ __align__(256) unsigned char g_noalloc_scratch[MBR_NOALLOC_SCRATCH_BYTES];

const size_t kGammaBytes = 65536 * sizeof(uint16_t);
const size_t kHeadBytes = kGammaBytes + 256;  // gamma table, then the status word

struct NoallocDevice {
  bool ready = false;
  unsigned char *base = nullptr;  // device address of g_noalloc_scratch on this device
  double gamma_value = -1.0;      // gamma of the table currently in the array
};
const int kMaxDevices = 64;
NoallocDevice g_noalloc[kMaxDevices];
std::mutex g_noalloc_mutex;
uint16_t g_noalloc_gamma_host[65536];  // host staging table of the gamma copies

mbr_status noalloc_fail(char *err, size_t err_len, mbr_status st, const std::string &msg) {
  if (err && err_len) std::snprintf(err, err_len, "%s", msg.c_str());
  return st;
}

// The largest pixel count whose scratch fits in `have` bytes.
long long noalloc_max_pixels(int per, size_t have) {
  const size_t per_pixel = sizeof(HitRec) + sizeof(float4) * (1 + size_t(per));
  long long n = (long long)((have - 256 - 255) / per_pixel);  // the hit region rounds up by < 256 bytes
  while (scratch_bytes(n + 1, per) <= have) n++;
  return n;
}

}  // namespace

extern "C" mbr_status mbr_render_noalloc(const mbr_scene *scene, const mbr_camera *camera,
                                         const mbr_render_params *params, const mbr_outputs *out, void *stream,
                                         char *err, size_t err_len) {
  if (err && err_len) err[0] = '\0';
  if (!scene || !camera || !params || !out) return noalloc_fail(err, err_len, MBR_EINVAL, "null argument");
  int dev = 0;
  int e = int(cudaGetDevice(&dev));
  if (e || dev < 0 || dev >= kMaxDevices)
    return noalloc_fail(err, err_len, MBR_ECUDA, "no current CUDA device");
  // one-time set-up on this device: the device address of the scratch array
  // (host code may not use the array's name as a device address)
  NoallocDevice *nd = &g_noalloc[dev];
  {
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!nd->ready) {
      void *ptr = nullptr;
      e = int(cudaGetSymbolAddress(&ptr, g_noalloc_scratch));
      if (e || !ptr)
        return noalloc_fail(err, err_len, MBR_ECUDA,
                            std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(cudaError_t(e)));
      nd->base = static_cast<unsigned char *>(ptr);
      nd->ready = true;
    }
  }
  DevScene sc;
  mbr_status st = build_scene(nullptr, *scene, &sc);
  if (st != MBR_OK) return noalloc_fail(err, err_len, st, "invalid or unsupported scene (see mbr_scene_set)");
  DevFrame fr;
  std::string msg;
  {
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);  // the host staging table is shared
    st = build_frame_owned_gamma(*camera, *params, reinterpret_cast<uint16_t *>(nd->base), g_noalloc_gamma_host,
                                 &nd->gamma_value, &fr, stream, &msg);
  }
  if (st != MBR_OK) return noalloc_fail(err, err_len, st, msg);
  fr.want_normal = out->normal != nullptr;
  if (sc.is_hybrid || sc.generic || sc.iter_thresh || sc.interior || sc.has_w || fr.gi_samples > 0 ||
      fr.refine != MBR_REFINE_REFERENCE || fr.slow_shading)
    return noalloc_fail(err, err_len, MBR_EUNSUPPORTED,
                        "the wavefront engine renders non-hybrid Mandelbulb, Mandelbox and Menger scenes without GI, "
                        "root refinement, iteration threshold, interior mode, initial w or slow shading");
  const long long total = (long long)fr.width * (fr.row1 - fr.row0);  // row-linear queue: no tile padding
  const int per = ((fr.shading_enable && fr.shadow_enable) ? 1 : 0) + ao_tasks(fr);
  const size_t need = scratch_bytes(total, per);
  const size_t have = size_t(MBR_NOALLOC_SCRATCH_BYTES) - kHeadBytes;
  if (need > have) {
    char buf[320];
    std::snprintf(buf, sizeof(buf),
                  "frame of %lld pixels with %d shadow/AO tasks per hit needs %zu bytes of scratch; the "
                  "allocation-free entry point has %zu (at most %lld pixels at this setting)",
                  total, per, need, have, noalloc_max_pixels(per, have));
    return noalloc_fail(err, err_len, MBR_EINVAL, buf);
  }
  Launch L;
  std::memset(&L, 0, sizeof(L));
  L.njobs = 1;
  L.total = total;
  scratch_layout(L, nd->base + kHeadBytes, total);
  const mbr_tuning tu{128, 12, 2, 0};
  L.refill_k = tu.refill_k;
  L.layout = tu.queue_layout;
  L.ao_rays = ao_tasks(fr);
  L.ao_fast = fr.ao_fast;
  L.shadow_tasks = (fr.shading_enable && fr.shadow_enable) ? 1 : 0;
  L.want_normal = fr.want_normal;
  DevOutputs d;
  d.depth = out->depth;
  d.iters = out->iters;
  d.hit = out->hit;
  d.normal = out->normal;
  d.shade = out->shade;
  d.ao = out->ao;
  d.rgb = out->rgb;
  d.rgb8 = out->rgb8;
  d.stats = out->stats;
  d.status = reinterpret_cast<int32_t *>(nd->base + kGammaBytes);
  d.pixel_offset = 0;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // the array keeps the previous call's contents: the status word starts at
  // zero here and the launch counters are zeroed at the head of the pipeline
  e = int(cudaMemsetAsync(d.status, 0, sizeof(int32_t), s));
  if (e) return noalloc_fail(err, err_len, MBR_ECUDA, std::string("cudaMemsetAsync: ") + cudaGetErrorString(cudaError_t(e)));
  const WJob j0 = make_job(fr, 0, 0);
  const FastParams fp = load_fast_params(sc);
  e = launch_pipeline<false, Prec32>(fast_kind(fp), tu, s, fr, fp, j0, L, d, total);
  if (e) return noalloc_fail(err, err_len, MBR_ECUDA, std::string("wavefront launch: ") + cudaGetErrorString(cudaError_t(e)));
  return MBR_OK;
}
