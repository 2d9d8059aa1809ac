// plain_kernel.cuh - the plain form: one thread per pixel running the whole
// per-pixel body of cRenderWorker::doWork (src/render_worker.cpp:126-525) for
// the level-0 ray: camera ray, march + refinement, normal, directional light
// with hard shadow, AO, or the Monte Carlo GI estimator with thin-lens DOF.
//
// Instantiated per translation unit with a variant tag V so that the FP64,
// strict-FP64 (no FMA contraction) and mixed-precision builds of the same
// template are distinct kernels.
#pragma once
#include "pixel_ops.cuh"

namespace mbr {

// One sample of the GI estimator (restated; see mbr.h): primary ray with MC
// pixel jitter and thin-lens DOF, direct sun with hard shadow at every
// vertex, cosine-sampled diffuse bounces marched with the GI rule.
template <class T, class R, int F, bool W>
__device__ double gi_path(const DevScene &sc, const DevFrame &fr, int x, int y, unsigned long long pixel, int sample,
                          ThreadCount &tc, MarchOut *first, unsigned int *n_march, unsigned int *n_binary,
                          unsigned int *n_gi) {
  const unsigned long long ray = pixel * (unsigned long long)fr.gi_samples + (unsigned long long)sample;
  Pcg32 rng = pcg_init(fr.gi_seed, ray);
  const double ujx = rng.uniform(), ujy = rng.uniform(), ulr = rng.uniform(), ula = rng.uniform();
  double ix, iy;
  image_point(fr, double(x), double(y), &ix, &iy);
  ix = ix + (ujx - 0.5) / double(fr.width) * fr.aspect;
  iy = iy + (ujy - 0.5) / double(fr.height);
  D3 view = view_vector(fr, ix, iy);
  const D3 cam = camera_of(fr);
  D3 start = cam;
  if (fr.dof_aperture > 0.0) {
    const double randR = fr.dof_aperture * sqrt(ulr);
    const double randAngle = 2.0 * 3.14159265358979323846 * ula;
    double sa, ca;
    sincos(randAngle, &sa, &ca);
    const D3 rv = rotate(fr, D3{randR * sa, 0.0, randR * ca});
    view = d3sub(view, d3mul(rv, 1.0 / fr.dof_focus));
    start = d3add(cam, rv);
  }
  const D3 dir = d3norm(view);
  ParkMiller pm = pm_for_ray(ray, fr.seed);
  const MarchOut m = ray_marching<T, R, F, W>(sc, fr, start, dir, pm, tc, n_march, n_binary);
  if (first) *first = m;
  const unsigned int de0 = tc.de;
  const D3 L{fr.light[0], fr.light[1], fr.light[2]};
  double radiance = 0.0, throughput = 1.0;
  if (!m.found) {
    radiance = fr.gi_sky;
  } else {
    D3 q = m.point;
    double thr = m.thr;
    D3 n = normals<T, F, W>(sc, fr, q, thr, tc);
    for (int bounce = 0;; bounce++) {
      const double ndl = d3dot(n, L);
      if (ndl > 0.0) {
        const double sh = aux_shadow<T, F, W>(sc, fr, q, thr, L, tc);
        radiance += throughput * double(fr.albedo) * fr.gi_sun * ndl * sh;
      }
      if (bounce >= fr.gi_bounces) break;
      throughput *= double(fr.albedo);
      const double u1 = rng.uniform(), u2 = rng.uniform();
      const D3 d = cosine_dir(n, u1, u2);
      bool found = false, ended = false;
      int steps = 0;
      double dist = 0.0;
      int it;
      for (double scan = thr; scan < fr.view_distance_max; scan += dist * fr.de_factor) {
        if (steps >= fr.max_steps) break;
        const D3 point = d3ray(q, d, scan);
        const double t2 = dist_thresh(sc, fr, point);
        dist = de_eval<T, F, W>(sc, point, t2, false, &it, tc);
        if (dist < t2) {
          if (scan < t2 * 2.0) {
            ended = true;
            break;
          }
          q = point;
          thr = t2;
          n = normals<T, F, W>(sc, fr, q, thr, tc);
          found = true;
          break;
        }
        steps++;
      }
      if (ended) break;
      if (!found) {
        radiance += throughput * fr.gi_sky;
        break;
      }
    }
  }
  *n_gi += tc.de - de0;
  return radiance;
}

template <class T, class R, int F, bool W, int V>
__global__ void __launch_bounds__(128) plain_kernel(const __grid_constant__ DevScene sc,
                                                    const __grid_constant__ DevFrame fr, DevOutputs out) {
  __shared__ unsigned long long cnt[K_COUNT];
  if (threadIdx.x < K_COUNT) cnt[threadIdx.x] = 0ull;
  __syncthreads();
  // a warp renders an 8x4 pixel tile, a block 16x8 pixels
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int x = blockIdx.x * 16 + (warp & 1) * 8 + (lane & 7);
  const int y = fr.row0 + blockIdx.y * 8 + (warp >> 1) * 4 + (lane >> 3);
  ThreadCount tc{0u, 0u};
  unsigned int n_march = 0, n_binary = 0, n_normal = 0, n_shadow = 0, n_ao = 0, n_gi = 0, trips = 0, n_pix = 0;
  if (x < fr.width && y < fr.row1) {
    const unsigned long long pixel = (unsigned long long)y * fr.width + x;
    MarchOut m;
    float nrm[3] = {0.0f, 0.0f, 0.0f};
    float shade = 0.0f, ao = 1.0f, rgb[3];
    double cx, cy;
    image_point(fr, double(x), double(y), &cx, &cy);
    if (hemisphere_cut(fr.persp, fr.fov, cx, cy)) {
      m.found = false;
      m.depth = 1e20;
      m.iters = 0;
      rgb[0] = rgb[1] = rgb[2] = 0.0f;
    } else if (fr.gi_samples > 0) {
      double acc = 0.0;
      for (int s = 0; s < fr.gi_samples; s++) {
        MarchOut mm;
        acc += gi_path<T, R, F, W>(sc, fr, x, y, pixel, s, tc, s == 0 ? &m : &mm, &n_march, &n_binary, &n_gi);
      }
      rgb[0] = rgb[1] = rgb[2] = float(acc / fr.gi_samples);
    } else {
      double ix, iy;
      image_point(fr, double(x), double(y), &ix, &iy);
      const D3 dir = d3norm(view_vector(fr, ix, iy));
      ParkMiller pm = pm_for_ray(pixel, fr.seed);
      m = ray_marching<T, R, F, W>(sc, fr, camera_of(fr), dir, pm, tc, &n_march, &n_binary);
      if (m.found) {
        D3 n{1.0, 0.0, 0.0};
        if (fr.shading_enable || fr.ao_rays > 0 || fr.ao_fast || fr.want_normal) {
          const unsigned int d0 = tc.de;
          n = normals<T, F, W>(sc, fr, m.point, m.thr, tc);
          n_normal += tc.de - d0;
          nrm[0] = float(n.x);
          nrm[1] = float(n.y);
          nrm[2] = float(n.z);
        }
        if (fr.shading_enable) {
          const D3 L{fr.light[0], fr.light[1], fr.light[2]};
          float s = float(d3dot(n, L));
          if (s < 0) s = 0;
          s = 1.0f - fr.material_shading + s * fr.material_shading;
          s = s * fr.light_intensity;
          if (s > 500.0f) s = 500.0f;
          float aux = 1.0f;
          if (fr.shadow_enable) {
            if (s > 0.001f) {
              const unsigned int d0 = tc.de;
              aux = float(aux_shadow<T, F, W>(sc, fr, m.point, m.thr, L, tc));
              n_shadow += tc.de - d0;
            } else {
              aux = 0.0f;
            }
          }
          shade = s * aux;
        }
        if (fr.ao_rays > 0 || fr.ao_fast) {
          const unsigned int d0 = tc.de;
          ao = float(ambient_occlusion<T, F, W>(sc, fr, m.point, n, m.thr, pixel, tc, &trips));
          n_ao += tc.de - d0;
        }
        const float col = fr.albedo * (shade + fr.ambient * ao);
        rgb[0] = rgb[1] = rgb[2] = col;
      } else {
        rgb[0] = fr.background[0];
        rgb[1] = fr.background[1];
        rgb[2] = fr.background[2];
      }
    }
    const long long o = out.pixel_offset + (long long)pixel;
    if (out.depth) out.depth[o] = m.found ? m.depth : 1e20;
    if (out.iters) out.iters[o] = m.iters;
    if (out.hit) out.hit[o] = m.found ? 1 : 0;
    if (out.normal) {
      out.normal[3 * o + 0] = nrm[0];
      out.normal[3 * o + 1] = nrm[1];
      out.normal[3 * o + 2] = nrm[2];
    }
    if (out.shade) out.shade[o] = shade;
    if (out.ao) out.ao[o] = ao;
    if (out.rgb) {
      out.rgb[3 * o + 0] = rgb[0];
      out.rgb[3 * o + 1] = rgb[1];
      out.rgb[3 * o + 2] = rgb[2];
    }
    if (out.rgb8) to_rgb8(fr, rgb, &out.rgb8[3 * o]);
    n_pix = 1;
  }
  if (out.status) {  // the watchdog status word: any AO march that reached its cap
    const unsigned int t = __reduce_add_sync(0xffffffffu, trips);
    if (lane == 0 && t) atomicOr(out.status, int(STATUS_AO_MARCH_CAP));
  }
  if (out.stats) {
    const unsigned int vals[K_COUNT] = {tc.de, tc.iters, n_march, n_binary, n_normal, n_shadow, n_ao, n_gi, n_pix, trips};
#pragma unroll
    for (int k = 0; k < K_COUNT; k++) {
      const unsigned int v = __reduce_add_sync(0xffffffffu, vals[k]);
      if (lane == 0 && v) atomicAdd(&cnt[k], (unsigned long long)v);
    }
    __syncthreads();
    if (threadIdx.x < K_COUNT && cnt[threadIdx.x])
      atomicAdd(reinterpret_cast<unsigned long long *>(out.stats) + threadIdx.x, cnt[threadIdx.x]);
  }
}

// CalculateDistance at n points (the reference's distance_engine.cl:42 job).
template <class T, int F, bool W, int V>
__global__ void __launch_bounds__(128) distance_kernel(const __grid_constant__ DevScene sc, const double *pts,
                                                       long long n, double detail, int normal_mode, double *dist,
                                                       int *iters) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  int it;
  const T d = calc_distance<T, F, W>(sc, T(pts[3 * i]), T(pts[3 * i + 1]), T(pts[3 * i + 2]), T(detail),
                                     normal_mode != 0, &it);
  dist[i] = double(d);
  if (iters) iters[i] = it;
}

template <class T, class R, int V>
int launch_plain_t(const DevScene &sc, const DevFrame &fr, const DevOutputs &out, void *stream) {
  const dim3 block(128);
  const dim3 grid((fr.width + 15) / 16, (fr.row1 - fr.row0 + 7) / 8);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const bool ext = scene_extended(sc) || fr.slow_shading;  // slow shading is compiled into F_EXT kernels only
  const int F = sc.is_hybrid ? 0 : sc.uniform_formula;
  if (sc.has_w) {
    if constexpr (sizeof(T) == 8) {
      if (ext) plain_kernel<T, R, F_EXT, true, V><<<grid, block, 0, s>>>(sc, fr, out);
      else plain_kernel<T, R, 0, true, V><<<grid, block, 0, s>>>(sc, fr, out);
    } else {
      return int(cudaErrorInvalidValue);
    }
  } else if (ext) {
    plain_kernel<T, R, F_EXT, false, V><<<grid, block, 0, s>>>(sc, fr, out);
  } else {
    switch (F) {
      case MBR_FORMULA_MANDELBULB: plain_kernel<T, R, MBR_FORMULA_MANDELBULB, false, V><<<grid, block, 0, s>>>(sc, fr, out); break;
      case MBR_FORMULA_MANDELBOX: plain_kernel<T, R, MBR_FORMULA_MANDELBOX, false, V><<<grid, block, 0, s>>>(sc, fr, out); break;
      case MBR_FORMULA_MENGER_SPONGE: plain_kernel<T, R, MBR_FORMULA_MENGER_SPONGE, false, V><<<grid, block, 0, s>>>(sc, fr, out); break;
      default: plain_kernel<T, R, 0, false, V><<<grid, block, 0, s>>>(sc, fr, out); break;
    }
  }
  return int(cudaGetLastError());
}

template <class T, int V>
int launch_distance_t(const DevScene &sc, const double *pts, int64_t n, double detail, int normal_mode, double *dist,
                      int32_t *iters, void *stream) {
  if (n <= 0) return 0;
  const dim3 block(128);
  const dim3 grid(unsigned((n + 127) / 128));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const bool ext = scene_extended(sc);
  if (sc.has_w) {
    if constexpr (sizeof(T) == 8) {
      if (ext) distance_kernel<T, F_EXT, true, V><<<grid, block, 0, s>>>(sc, pts, n, detail, normal_mode, dist, iters);
      else distance_kernel<T, 0, true, V><<<grid, block, 0, s>>>(sc, pts, n, detail, normal_mode, dist, iters);
    } else {
      return int(cudaErrorInvalidValue);
    }
  } else if (ext) {
    distance_kernel<T, F_EXT, false, V><<<grid, block, 0, s>>>(sc, pts, n, detail, normal_mode, dist, iters);
  } else {
    distance_kernel<T, 0, false, V><<<grid, block, 0, s>>>(sc, pts, n, detail, normal_mode, dist, iters);
  }
  return int(cudaGetLastError());
}

}  // namespace mbr
