// wavefront.cu - the batched FP32 form.
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
//   stage S  (1 + ao_rays) tasks per hit: the hard AuxShadow march
//            (src/shader_aux_shadow.cpp:94-321) and one AmbientOcclusion
//            march per AO direction (src/shader_ambient_occlusion.cpp:60-110)
//   stage F  one thread per hit: colour, 8-bit conversion, outputs
//
// Every march is a stream of distance requests p = origin + dir * t with t
// and the origin in FP64 and the formula iteration in FP32.  In stages P, N
// and S each lane holds one task; it runs two formula iterations between
// warp votes and, once at most k lanes of the warp are still iterating, the
// lanes whose estimate is done take their march step and start their next
// request, or take the next task from the stage's device counter
// (warp-aggregated atomicAdd).  Because a warp only ever runs one kind of
// march, those steps stay converged and cheap, and divergent orbit lengths
// and march lengths cost only the k-lane wait.  A batch walks a job table
// (per-job camera, image size and formula parameters) with the same stages,
// captured once into a CUDA graph.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "fast_formula.cuh"
#include "fastdiv.h"
#include "mbr_internal.h"
#include "pixel_ops.cuh"

namespace mbr {

// formula kinds of the iteration switch
enum { FK_ANY = 0, FK_BULB = 2, FK_MENGER = 7, FK_BOX = 8, FK_BOX_SIMPLE = 108 };

// One render job of a launch: its camera, image size and place in the queue.
struct WJob {
  double cam[3];
  double mrot[9];
  int32_t mrot_zero;
  int32_t width, height, tiles_x;
  int32_t row0, rows;      // the job renders rows [row0, row0 + rows) of its frame
  long long first;         // first work item of this job in the pixel queue
  long long pixel_offset;  // first pixel of this job in the outputs
  double fov, aspect;
  float c0;                // threshold per unit distance: resolution * fov / detail
  float fovf;              // fov (AO end distance = |camera - p| * fov)
  FastDiv div_w, div_tx;   // divisions by width and tiles_x
};

// A surface hit, produced by stage P and completed by stages N and S.
struct HitRec {
  double px, py, pz;  // hit point
  double depth;       // scan distance t of the hit
  long long pix;      // output index
  float thr;          // distThresh at the hit
  int iters;          // iters of the last primary DE evaluation
  float nx, ny, nz;   // normal
  float shade;        // Lambert term before the shadow
  float shadow;       // AuxShadow result
  int job;
  unsigned int ray;   // pixel index within its job (RNG streams)
  int pad;
  // sum of the AO march results in 32.32 fixed point: integer atomics make
  // the sum independent of the order in which the AO marches finish
  unsigned long long ao_q;
};

__device__ __forceinline__ void ao_add(HitRec *r, float s) {
  atomicAdd(&r->ao_q, (unsigned long long)(double(s) * 4294967296.0));
}

// Device-side counters of one launch (in the context's scratch).
struct Counters4 {
  unsigned long long pixels_next;  // stage P queue
  unsigned long long hits;         // hits appended by stage P
  unsigned long long normals_next; // stage N queue
  unsigned long long shade_next;   // stage S queue
};

struct Launch {
  const WJob *jobs;        // njobs entries (device)
  const FastParams *fps;   // per job (device)
  int njobs;
  long long total;         // pixel work items
  HitRec *hits;            // capacity: total
  float4 *sorg;            // per hit: FP32 hit point and threshold (stage S origins)
  float4 *sdir;            // per stage-S task: direction and end (w < 0: shadow, w == 0: no march)
  Counters4 *ctr;
  int refill_k;
  int layout;
  int ao_rays;
  int shadow_tasks;        // 1 when the shadow march runs (shading && shadow)
  int want_normal;
  FastDiv div_per;         // division by shadow_tasks + ao_rays (set by launch_pipeline)
};

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

template <int FK>
__device__ __forceinline__ void iterate(int kind, Z3 &z, float &dr, const Z3 &c, const FastParams &f, float r2) {
  const int k = (FK == FK_ANY) ? kind : FK;
  if (k == FK_BOX_SIMPLE) it_mandelbox<true>(z, dr, c, f);
  else if (k == FK_BOX) it_mandelbox<false>(z, dr, c, f);
  else if (k == FK_BULB) it_mandelbulb(z, dr, c, f, sqrtf(r2));
  else it_menger(z, dr, c, f);
}

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

// Per-lane state of one distance estimate.
struct DE {
  Z3 z, c;
  float dr, r2;
  int it;
};

__device__ __forceinline__ void de_start(DE &e, const FastParams &fp, double qx, double qy, double qz) {
  e.z.x = float(qx);
  e.z.y = float(qy);
  e.z.z = float(qz);
  if (!fp.add_c) e.c = Z3{0.f, 0.f, 0.f};
  else if (fp.julia) e.c = Z3{fp.jc_x, fp.jc_y, fp.jc_z};
  else e.c = Z3{e.z.x * fp.cm_x, e.z.y * fp.cm_y, e.z.z * fp.cm_z};
  e.dr = 1.f;
  e.it = 0;
  e.r2 = fmaf(e.z.x, e.z.x, fmaf(e.z.y, e.z.y, e.z.z * e.z.z));
}

__device__ __forceinline__ void de_start(DE &e, const FastParams &fp, float qx, float qy, float qz) {
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

// ============================================================================
// The persistent skeleton: refill lanes from a task counter, iterate, step.
// Stage provides (Real: the precision of its request points):
//   bool start(long long task, Real &qx, &qy, &qz)   - first request (false: nothing to march)
//   bool step(float d, int iters, Real &qx, &qy, &qz) - consume a result; true: next request
//   const FastParams &params()  - formula of the current task
//   int kind()                  - formula kind (FK_ANY launches)
// ============================================================================
template <int FK, class Stage>
__device__ __forceinline__ void run_stage(Stage &S, unsigned long long *counter, long long total, int refill_k,
                                          unsigned int *my_de, unsigned long long *my_iters) {
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const unsigned lanemask_lt = (1u << lane) - 1u;
  DE e;
  e.it = 0;
  e.r2 = 0.f;
  e.dr = 1.f;
  bool has = false, iterating = false, drained = false;
  unsigned int de_n = 0;
  unsigned long long it_n = 0;
  for (;;) {
    // ---- refill lanes without a task
    unsigned need = __ballot_sync(FULL, !has && !drained);
    while (need) {
      const int leader = __ffs(need) - 1;
      unsigned long long base = 0ull;
      if (lane == leader) base = atomicAdd(counter, (unsigned long long)__popc(need));
      base = __shfl_sync(FULL, base, leader);
      bool empty = false;
      if (!has && !drained) {
        const long long idx = (long long)base + (long long)__popc(need & lanemask_lt);
        if (idx < total) {
          typename Stage::Real qx, qy, qz;
          if (S.start(idx, qx, qy, qz)) {
            de_start(e, S.params(), qx, qy, qz);
            has = true;
            iterating = true;
          }
        } else {
          empty = true;
        }
      }
      if (__any_sync(FULL, empty)) drained = true;
      need = __ballot_sync(FULL, !has && !drained);
    }
    if (!__any_sync(FULL, iterating)) break;
    const int k = drained ? 0 : refill_k;
    // ---- formula iterations, two between votes, until <= k lanes still iterate.
    // A lane whose orbit ends leaves the loop by a branch, so the remaining
    // lanes run the iteration without select instructions for finished ones;
    // the vote counts the lanes still in the loop.
    const FastParams &fp = S.params();
    const int kind = S.kind();
    if (iterating) {
      for (;;) {
        iterate<FK>(kind, e.z, e.dr, e.c, fp, e.r2);
        e.it++;
        e.r2 = fmaf(e.z.x, e.z.x, fmaf(e.z.y, e.z.y, e.z.z * e.z.z));
        if (!(e.r2 <= fp.bailout2) || e.it >= fp.maxN) {
          iterating = false;
          break;
        }
        iterate<FK>(kind, e.z, e.dr, e.c, fp, e.r2);
        e.it++;
        e.r2 = fmaf(e.z.x, e.z.x, fmaf(e.z.y, e.z.y, e.z.z * e.z.z));
        if (!(e.r2 <= fp.bailout2) || e.it >= fp.maxN) {
          iterating = false;
          break;
        }
        if (!more_than(__ballot_sync(__activemask(), 1), k)) break;
      }
    }
    __syncwarp();
    // ---- lanes whose estimate is done: distance, then the march step
    if (has && !iterating) {
      const bool bailed = e.r2 > fp.bailout2;
      const int iters = bailed ? e.it : e.it + 1;
      const float d = final_de(fp, e.r2, e.dr, iters, S.detail());
      de_n++;
      it_n += (unsigned long long)iters;
      typename Stage::Real qx, qy, qz;
      if (S.step(d, iters, qx, qy, qz)) {
        de_start(e, S.params(), qx, qy, qz);
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
template <bool MULTI>
struct PrimaryStage {
  typedef double Real;
  const DevFrame &fr;
  const Launch &L;
  const DevOutputs &out;
  const WJob *jb;
  FastParams fp;
  int kd;
  int job;
  // ray
  double dx, dy, dz, ox, oy, oz, t, stp;
  float thr, c0, dist_prev, search_limit;
  int phase, sub, count, last_iters;
  unsigned int pm, ray, binary_de;
  long long pix;

  __device__ const FastParams &params() const { return fp; }
  __device__ int kind() const { return kd; }
  __device__ float detail() const { return thr; }

  __device__ void point(double &qx, double &qy, double &qz) {
    thr = fr.constant_de_threshold ? float(fr.de_thresh) : float(t) * c0;
    qx = fma(dx, t, ox);
    qy = fma(dy, t, oy);
    qz = fma(dz, t, oz);
  }

  __device__ bool start(long long idx, double &qx, double &qy, double &qz) {
    if (MULTI) {
      job = job_of(L.jobs, L.njobs, idx);
      jb = &L.jobs[job];
      fp = L.fps[job];
      kd = fast_kind(fp);
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
    const double iy = -1.0 / double(jb->height) * double(y) + 0.5;
    double vx = ix * jb->fov, vy = 1.0, vz = iy * jb->fov;
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
    ox = jb->cam[0];
    oy = jb->cam[1];
    oz = jb->cam[2];
    c0 = jb->c0;
    t = 0.0;
    stp = 0.0;
    phase = 0;
    sub = 0;
    count = 0;
    last_iters = 0;
    if (fr.jitter) pm = pm_for_ray(ray, fr.seed).s;
    point(qx, qy, qz);
    return true;
  }

  __device__ void write_miss() {
    float rgb[3] = {fr.background[0], fr.background[1], fr.background[2]};
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
    r.thr = thr;
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

  __device__ bool step(float d, int iters, double &qx, double &qy, double &qz) {
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
    stp = double((d - 0.5f * thr) * float(fr.de_factor)) * jit;
    if (stp > 3.0) stp = 3.0;
    t += stp;
    if (t > fr.view_distance_max || count >= fr.max_steps) {
      write_miss();
      return false;
    }
    point(qx, qy, qz);
    return true;
  }
};

template <int FK, bool MULTI>
__global__ void __launch_bounds__(256) primary_kernel(const __grid_constant__ DevFrame fr,
                                                      const __grid_constant__ FastParams fp0,
                                                      const __grid_constant__ WJob job0,
                                                      const __grid_constant__ Launch L, DevOutputs out) {
  PrimaryStage<MULTI> S{fr, L, out, &job0, fp0, fast_kind(fp0), 0};
  S.search_limit = float(1.0 - 0.001 * fr.detail_level);
  S.binary_de = 0;
  unsigned int my_de = 0;
  unsigned long long my_iters = 0;
  run_stage<FK>(S, &L.ctr->pixels_next, L.total, L.refill_k, &my_de, &my_iters);
  flush_counts(out, my_de, my_iters, K_MARCH, my_de - S.binary_de, K_BINARY, S.binary_de);
}

// ============================================================================
// Stage N: normals + Lambert term, one task per hit.
// ============================================================================
template <bool MULTI>
struct NormalStage {
  typedef double Real;
  const DevFrame &fr;
  const Launch &L;
  FastParams fp;
  int kd;
  HitRec *r;
  double ox, oy, oz, delta;
  float thr, nx, ny, nz;
  int sub;

  __device__ const FastParams &params() const { return fp; }
  __device__ int kind() const { return kd; }
  __device__ float detail() const { return thr; }

  __device__ void point(double &qx, double &qy, double &qz) {
    const double dd = (sub & 1) ? -delta : delta;
    const int axis = sub >> 1;
    qx = ox + (axis == 0 ? dd : 0.0);
    qy = oy + (axis == 1 ? dd : 0.0);
    qz = oz + (axis == 2 ? dd : 0.0);
  }

  __device__ bool start(long long idx, double &qx, double &qy, double &qz) {
    r = &L.hits[idx];
    if (MULTI) {
      fp = L.fps[r->job];
      kd = fast_kind(fp);
    }
    ox = r->px;
    oy = r->py;
    oz = r->pz;
    thr = r->thr;
    delta = double(thr) * fr.smoothness;
    sub = 0;
    nx = ny = nz = 0.f;
    point(qx, qy, qz);
    return true;
  }

  __device__ bool step(float d, int, double &qx, double &qy, double &qz) {
    const bool neg = (sub & 1) != 0;
    const int axis = sub >> 1;
    float &comp = (axis == 0) ? nx : ((axis == 1) ? ny : nz);
    comp = neg ? comp - d : d;
    sub++;
    if (sub < 6) {
      point(qx, qy, qz);
      return true;
    }
    // CalculateNormals tail (shader_calculate_normals.cpp:111-123)
    if (fabsf(nx) < 1e-30f && fabsf(ny) < 1e-30f && fabsf(nz) < 1e-30f) {
      nx = 1.f;
      ny = nz = 0.f;
    } else {
      const float inv = rsqrtf(nx * nx + ny * ny + nz * nz);
      nx *= inv;
      ny *= inv;
      nz *= inv;
    }
    if (!(isfinite(nx) && isfinite(ny) && isfinite(nz))) {
      nx = 1.f;
      ny = nz = 0.f;
    }
    r->nx = nx;
    r->ny = ny;
    r->nz = nz;
    // LightShading, directional light (shader_light_shading.cpp:61-72)
    float s = 0.f;
    if (fr.shading_enable) {
      s = nx * float(fr.light[0]) + ny * float(fr.light[1]) + nz * float(fr.light[2]);
      if (s < 0) s = 0;
      s = 1.0f - fr.material_shading + s * fr.material_shading;
      s = s * fr.light_intensity;
      if (s > 500.0f) s = 500.0f;
    }
    r->shade = s;
    return false;
  }
};

template <int FK, bool MULTI>
__global__ void __launch_bounds__(256) normal_kernel(const __grid_constant__ DevFrame fr,
                                                     const __grid_constant__ FastParams fp0,
                                                     const __grid_constant__ Launch L, DevOutputs out) {
  NormalStage<MULTI> S{fr, L, fp0, fast_kind(fp0)};
  unsigned int my_de = 0;
  unsigned long long my_iters = 0;
  const long long total = (long long)L.ctr->hits;
  run_stage<FK>(S, &L.ctr->normals_next, total, L.refill_k, &my_de, &my_iters);
  flush_counts(out, my_de, my_iters, K_NORMAL, my_de, K_NORMAL, 0);
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

template <bool MULTI>
struct ShadeStage {
  // secondary rays start at the FP64 hit point, rounded once to FP32; their
  // march runs in FP32 (no FP64 conversions in the loop)
  typedef float Real;
  const DevFrame &fr;
  const Launch &L;
  FastParams fp;
  int kd;
  HitRec *r;
  float ox, oy, oz, t;
  float dx, dy, dz, thr, end, vdm, dfac;
  int count, mode;  // mode 0 shadow, 1 AO
  unsigned int shadow_de;

  __device__ const FastParams &params() const { return fp; }
  __device__ int kind() const { return kd; }
  __device__ float detail() const { return thr; }

  __device__ void point(float &qx, float &qy, float &qz) {
    qx = fmaf(dx, t, ox);
    qy = fmaf(dy, t, oy);
    qz = fmaf(dz, t, oz);
  }

  __device__ bool start(long long idx, float &qx, float &qy, float &qz) {
    const float4 dv = L.sdir[idx];
    if (dv.w == 0.0f) return false;  // resolved by the direction kernel
    const long long h = (long long)fdiv((unsigned long long)idx, L.div_per);
    r = &L.hits[h];
    if (MULTI) {
      fp = L.fps[r->job];
      kd = fast_kind(fp);
    }
    const float4 o = L.sorg[h];
    ox = o.x;
    oy = o.y;
    oz = o.z;
    thr = o.w;
    dx = dv.x;
    dy = dv.y;
    dz = dv.z;
    mode = dv.w < 0.0f ? 0 : 1;
    end = mode ? dv.w : vdm;
    count = 0;
    t = thr;
    point(qx, qy, qz);
    return true;
  }

  __device__ bool step(float d, int, float &qx, float &qy, float &qz) {
    count++;
    if (mode == 0) {
      shadow_de++;
      if (d < thr) {
        r->shadow = 0.f;
        return false;
      }
      t += fmaxf(fminf(d, 1e6f) * dfac, 1e-15f);
      if (count > fr.max_steps || t >= vdm) {
        r->shadow = 1.f;
        return false;
      }
    } else {
      if (d < thr) {
        const float s = 1.0f - __fdividef(end - t, end);
        ao_add(r, fmaxf(s, 0.0f));
        return false;
      }
      t = fmaf(2.0f, d, t);
      if (t >= end || count >= fr.max_steps) {
        ao_add(r, 1.0f);
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
  const long long nh = (long long)L.ctr->hits;
  const int per = L.shadow_tasks + L.ao_rays;
  const long long n = nh * per;
  const float vdm = float(fr.view_distance_max);
  for (long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x; idx < n;
       idx += (long long)gridDim.x * blockDim.x) {
    const long long h = (long long)fdiv((unsigned long long)idx, L.div_per);
    const int k = int(idx - h * per);
    HitRec &r = L.hits[h];
    const float thr = r.thr;
    if (k == 0) L.sorg[h] = make_float4(float(r.px), float(r.py), float(r.pz), thr);
    float4 dv;
    if (k < L.shadow_tasks) {
      if (!(r.shade > 0.001f)) {
        r.shadow = 0.f;
        dv = make_float4(0.f, 0.f, 0.f, 0.f);
      } else if (!(thr < vdm)) {
        r.shadow = 1.f;
        dv = make_float4(0.f, 0.f, 0.f, 0.f);
      } else {
        dv = make_float4(float(fr.light[0]), float(fr.light[1]), float(fr.light[2]), -1.0f);
      }
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
        ao_add(&r, 1.0f);  // no room to march: unoccluded
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

template <int FK, bool MULTI>
__global__ void __launch_bounds__(256) shade_kernel(const __grid_constant__ DevFrame fr,
                                                    const __grid_constant__ FastParams fp0,
                                                    const __grid_constant__ Launch L, DevOutputs out) {
  ShadeStage<MULTI> S{fr, L, fp0, fast_kind(fp0)};
  S.shadow_de = 0;
  S.vdm = float(fr.view_distance_max);
  S.dfac = float(fr.de_factor);
  unsigned int my_de = 0;
  unsigned long long my_iters = 0;
  const long long total = (long long)L.ctr->hits * (long long)(L.shadow_tasks + L.ao_rays);
  run_stage<FK>(S, &L.ctr->shade_next, total, L.refill_k, &my_de, &my_iters);
  flush_counts(out, my_de, my_iters, K_AO, my_de - S.shadow_de, K_SHADOW, S.shadow_de);
}

// ============================================================================
// Stage F: colour and outputs of every hit.
// ============================================================================
__global__ void __launch_bounds__(256) finish_kernel(const __grid_constant__ DevFrame fr,
                                                     const __grid_constant__ Launch L, DevOutputs out) {
  const long long nh = (long long)L.ctr->hits;
  for (long long h = (long long)blockIdx.x * blockDim.x + threadIdx.x; h < nh; h += (long long)gridDim.x * blockDim.x) {
    const HitRec &r = L.hits[h];
    const long long pix = r.pix;
    const float shade = r.shade * r.shadow;
    const float ao = (L.ao_rays > 0) ? float(double(r.ao_q) * (1.0 / 4294967296.0) / double(L.ao_rays)) : 1.0f;
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
  if (threadIdx.x == 0 && out.stats) atomicAdd(reinterpret_cast<unsigned long long *>(out.stats) + K_PIXELS,
                                               (unsigned long long)pixels);
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
  j.aspect = fr.aspect;
  j.c0 = float(fr.resolution * fr.fov / fr.detail_level);
  j.fovf = float(fr.fov);
  j.div_w = make_fastdiv(j.width);
  j.div_tx = make_fastdiv(j.tiles_x);
  return j;
}

static long long job_items(const WJob &j, int layout) {
  if (layout == 1) return (long long)j.tiles_x * ((j.rows + 3) / 4) * 32;
  return (long long)j.width * j.rows;
}

static mbr_status check_supported(mbr_ctx *ctx, const DevScene &sc, const DevFrame &fr) {
  if (sc.is_hybrid) return set_err(ctx, MBR_EUNSUPPORTED, "wavefront engine: hybrid sequences use the plain engines");
  if (sc.iter_thresh || sc.interior || sc.has_w)
    return set_err(ctx, MBR_EUNSUPPORTED,
                   "wavefront engine: iteration_threshold_mode, interior_mode and initial_waxis != 0 use the plain engines");
  if (fr.gi_samples > 0 || fr.refine != MBR_REFINE_REFERENCE)
    return set_err(ctx, MBR_EUNSUPPORTED, "wavefront engine: GI and root refinement use the plain engines");
  return MBR_OK;
}

static int sm_count() {
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  return sms;
}

// The stage launches of one frame or batch, in stream order.
template <bool MULTI>
static int launch_pipeline(int fk, const mbr_tuning &tu, cudaStream_t st, const DevFrame &fr, const FastParams &fp0,
                           const WJob &j0, const Launch &L0, const DevOutputs &out, long long pixels) {
  Launch L = L0;
  L.div_per = make_fastdiv(std::max(1, L.shadow_tasks + L.ao_rays));
  const int sms = sm_count();
  const int grid = std::max(1, sms * tu.ctas_per_sm);
  const int block = tu.block_size;
  int e = int(cudaMemsetAsync(L.ctr, 0, sizeof(Counters4), st));
  if (e) return e;
#define STAGE_LAUNCH(KERNEL, K, ...)                                                    \
  case K:                                                                               \
    KERNEL<K, MULTI><<<grid, block, 0, st>>>(__VA_ARGS__);                              \
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
    STAGE(shade_kernel, fr, fp0, L, out)
  }
#undef STAGE
#undef STAGE_LAUNCH
  finish_kernel<<<sms * 4, 256, 0, st>>>(fr, L, out);
  pixel_count_kernel<<<1, 32, 0, st>>>(L, out, pixels);
  return int(cudaGetLastError());
}

// Scratch of a launch over `pixels` work items with `per` stage-S tasks per
// hit: counters, hit records, FP32 origins and stage-S start records.
static size_t scratch_bytes(long long pixels, int per) {
  return 256 + size_t(pixels) * (sizeof(HitRec) + sizeof(float4) * (1 + size_t(per)));
}

static void scratch_layout(Launch &L, void *base, long long pixels) {
  char *p = static_cast<char *>(base);
  L.ctr = reinterpret_cast<Counters4 *>(p);
  L.hits = reinterpret_cast<HitRec *>(p + 256);
  L.sorg = reinterpret_cast<float4 *>(p + 256 + size_t(pixels) * sizeof(HitRec));
  L.sdir = L.sorg + pixels;
}

mbr_status render_wavefront(mbr_ctx *ctx, const DevScene &sc, const DevFrame &fr, const DevOutputs &out, int engine,
                            void *stream) {
  if (engine != MBR_ENGINE_WAVEFRONT_FP32)
    return set_err(ctx, MBR_EUNSUPPORTED, "the FP64 wavefront engine is not built; use MBR_ENGINE_PLAIN_FP64");
  mbr_status stt = check_supported(ctx, sc, fr);
  if (stt != MBR_OK) return stt;
  const mbr_tuning tu = ctx_tuning(ctx);
  const WJob j0 = make_job(fr, 0, out.pixel_offset);
  const long long total = job_items(j0, tu.queue_layout);
  const int per = ((fr.shading_enable && fr.shadow_enable) ? 1 : 0) + fr.ao_rays;
  const size_t bytes = scratch_bytes(total, per);
  unsigned long long *work = nullptr;
  stt = ctx_work(ctx, (bytes + 7) / 8, &work);
  if (stt != MBR_OK) return stt;
  Launch L;
  std::memset(&L, 0, sizeof(L));
  L.jobs = nullptr;
  L.fps = nullptr;
  L.njobs = 1;
  L.total = total;
  scratch_layout(L, work, total);
  L.refill_k = tu.refill_k;
  L.layout = tu.queue_layout;
  L.ao_rays = fr.ao_rays;
  L.shadow_tasks = (fr.shading_enable && fr.shadow_enable) ? 1 : 0;
  L.want_normal = fr.want_normal;
  const FastParams fp = load_fast_params(sc);
  const int e = launch_pipeline<false>(fast_kind(fp), tu, static_cast<cudaStream_t>(stream), fr, fp, j0, L, out,
                                       (long long)fr.width * (fr.row1 - fr.row0));
  return cuda_err(ctx, e, "wavefront launch");
}

}  // namespace mbr

// ============================================================================
// Batches and the autotuner
// ============================================================================
using namespace mbr;

struct mbr_batch {
  mbr_ctx *ctx = nullptr;
  WJob *d_jobs = nullptr;
  FastParams *d_params = nullptr;
  void *d_scratch = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  long long total = 0;
};

extern "C" {

mbr_status mbr_batch_create(mbr_ctx *ctx, const mbr_scene *scenes, int32_t n_scenes, const mbr_job *jobs,
                            int32_t n_jobs, const mbr_render_params *params, const mbr_outputs *outs, int engine,
                            void *stream, mbr_batch **batch) {
  if (!batch) return set_err(ctx, MBR_EINVAL, "null batch pointer");
  *batch = nullptr;
  if (!ctx || !scenes || !jobs || !params || !outs || n_scenes < 1 || n_jobs < 1)
    return set_err(ctx, MBR_EINVAL, "null argument or empty batch");
  if (engine != MBR_ENGINE_WAVEFRONT_FP32)
    return set_err(ctx, MBR_EUNSUPPORTED, "batches run on MBR_ENGINE_WAVEFRONT_FP32");
  const mbr_tuning tu = ctx_tuning(ctx);
  std::vector<FastParams> fps(n_jobs);
  std::vector<WJob> wj(n_jobs);
  std::vector<DevScene> dsc(n_scenes);
  for (int i = 0; i < n_scenes; i++) {
    mbr_status st = build_scene(ctx, scenes[i], &dsc[i]);
    if (st != MBR_OK) return st;
  }
  DevFrame fr0;
  long long first = 0, pixels = 0;
  for (int i = 0; i < n_jobs; i++) {
    const mbr_job &jb = jobs[i];
    if (jb.scene_index < 0 || jb.scene_index >= n_scenes)
      return set_err(ctx, MBR_EINVAL, "job %d: scene_index %d out of range", i, jb.scene_index);
    if (jb.pixel_offset < 0) return set_err(ctx, MBR_EINVAL, "job %d: negative pixel_offset", i);
    DevFrame fr;
    mbr_status st = build_frame(ctx, jb.camera, *params, &fr);
    if (st != MBR_OK) return st;
    st = check_supported(ctx, dsc[jb.scene_index], fr);
    if (st != MBR_OK) return st;
    if (i == 0) fr0 = fr;
    wj[i] = make_job(fr, first, jb.pixel_offset);
    first += job_items(wj[i], tu.queue_layout);
    pixels += (long long)fr.width * (fr.row1 - fr.row0);
    fps[i] = load_fast_params(dsc[jb.scene_index]);
  }
  fr0.want_normal = outs->normal != nullptr;
  mbr_batch *b = new mbr_batch();
  b->ctx = ctx;
  b->total = first;
  auto fail = [&](int e, const char *what) {
    mbr_batch_destroy(b);
    return cuda_err(ctx, e, what);
  };
  int e = int(cudaMalloc(&b->d_jobs, sizeof(WJob) * n_jobs));
  if (e) return fail(e, "cudaMalloc(jobs)");
  e = int(cudaMalloc(&b->d_params, sizeof(FastParams) * n_jobs));
  if (e) return fail(e, "cudaMalloc(params)");
  const int per = ((fr0.shading_enable && fr0.shadow_enable) ? 1 : 0) + fr0.ao_rays;
  e = int(cudaMalloc(&b->d_scratch, scratch_bytes(first, per)));
  if (e) return fail(e, "cudaMalloc(scratch)");
  e = int(cudaMemcpy(b->d_jobs, wj.data(), sizeof(WJob) * n_jobs, cudaMemcpyHostToDevice));
  if (e) return fail(e, "cudaMemcpy(jobs)");
  e = int(cudaMemcpy(b->d_params, fps.data(), sizeof(FastParams) * n_jobs, cudaMemcpyHostToDevice));
  if (e) return fail(e, "cudaMemcpy(params)");
  Launch L;
  std::memset(&L, 0, sizeof(L));
  L.jobs = b->d_jobs;
  L.fps = b->d_params;
  L.njobs = n_jobs;
  L.total = first;
  scratch_layout(L, b->d_scratch, first);
  L.refill_k = tu.refill_k;
  L.layout = tu.queue_layout;
  L.ao_rays = fr0.ao_rays;
  L.shadow_tasks = (fr0.shading_enable && fr0.shadow_enable) ? 1 : 0;
  L.want_normal = fr0.want_normal;
  // capture the pipeline of one batch into a graph
  cudaStream_t cs;
  e = int(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
  if (e) return fail(e, "cudaStreamCreate");
  const DevOutputs d = dev_outputs(ctx, *outs);
  e = int(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal));
  if (!e) {
    const int le = launch_pipeline<true>(FK_ANY, tu, cs, fr0, fps[0], wj[0], L, d, pixels);
    cudaGraph_t g = nullptr;
    e = int(cudaStreamEndCapture(cs, &g));
    b->graph = g;
    if (!e) e = le;
  }
  cudaStreamDestroy(cs);
  if (e) return fail(e, "graph capture");
  e = int(cudaGraphInstantiate(&b->exec, b->graph, 0));
  if (e) return fail(e, "cudaGraphInstantiate");
  (void)stream;
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
  if (b->d_scratch) cudaFree(b->d_scratch);
  delete b;
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
  float best_ms = 1e30f;
  mbr_tuning bt = saved;
  const int blocks[] = {128, 256};  // __launch_bounds__(256)
  const int ctas[] = {6, 8, 12};
  const int ks[] = {0, 2, 4, 8, 16, 24};
  const int layouts[] = {0, 1};
  mbr_status status = MBR_OK;
  for (int b : blocks)
    for (int c : ctas) {
      if (b * c > 2048) continue;
      for (int k : ks)
        for (int l : layouts) {
          mbr_tuning t{b, c, k, l};
          ctx_tuning(ctx) = t;
          status = mbr_render(ctx, camera, params, out, engine, stream);  // warm-up
          if (status != MBR_OK) goto done;
          cudaEventRecord(e0, st);
          status = mbr_render(ctx, camera, params, out, engine, stream);
          cudaEventRecord(e1, st);
          if (status != MBR_OK) goto done;
          cudaEventSynchronize(e1);
          float ms = 0.f;
          cudaEventElapsedTime(&ms, e0, e1);
          if (ms < best_ms) {
            best_ms = ms;
            bt = t;
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

mbr_status noalloc_fail(char *err, size_t err_len, mbr_status st, const std::string &msg) {
  if (err && err_len) std::snprintf(err, err_len, "%s", msg.c_str());
  return st;
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
  st = build_frame_owned_gamma(*camera, *params, reinterpret_cast<uint16_t *>(nd->base), &nd->gamma_value, &fr,
                               &msg);
  if (st != MBR_OK) return noalloc_fail(err, err_len, st, msg);
  fr.want_normal = out->normal != nullptr;
  if (sc.is_hybrid || sc.iter_thresh || sc.interior || sc.has_w || fr.gi_samples > 0 ||
      fr.refine != MBR_REFINE_REFERENCE)
    return noalloc_fail(err, err_len, MBR_EUNSUPPORTED,
                        "the wavefront engine renders non-hybrid scenes without GI, root refinement, "
                        "iteration threshold, interior mode or initial w");
  const long long total = (long long)fr.width * (fr.row1 - fr.row0);  // row-linear queue: no tile padding
  const int per = ((fr.shading_enable && fr.shadow_enable) ? 1 : 0) + fr.ao_rays;
  const size_t need = scratch_bytes(total, per);
  const size_t have = size_t(MBR_NOALLOC_SCRATCH_BYTES) - kHeadBytes;
  if (need > have) {
    const size_t per_pixel = sizeof(HitRec) + sizeof(float4) * (1 + size_t(per));
    char buf[320];
    std::snprintf(buf, sizeof(buf),
                  "frame of %lld pixels with %d shadow/AO tasks per hit needs %zu bytes of scratch; the "
                  "allocation-free entry point has %zu (at most %zu pixels at this setting)",
                  total, per, need, have, (have - 256) / per_pixel);
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
  L.ao_rays = fr.ao_rays;
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
  e = launch_pipeline<false>(fast_kind(fp), tu, s, fr, fp, j0, L, d, total);
  if (e) return noalloc_fail(err, err_len, MBR_ECUDA, std::string("wavefront launch: ") + cudaGetErrorString(cudaError_t(e)));
  return MBR_OK;
}
