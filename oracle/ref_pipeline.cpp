// ref_pipeline.cpp - C entry points around the REFERENCE's own compiled
// sources for the whole distance-estimation path: the parameter containers
// with the reference's defaults (src/initparameters.cpp), the objects tree
// (src/objects_tree.cpp), sParamRender (src/fractparams.cpp), the hybrid
// sequences (src/hybrid_fractal_sequences.cpp), Compute
// (src/compute_fractal.cpp), CalculateDistance (src/calculate_distance.cpp),
// every formula of formula/definition/, and cRenderWorker::doWork
// (src/render_worker.cpp) with its shaders (src/shader_*.cpp) into a cImage
// (src/cimage.cpp).  Built by oracle/build_ref.sh into
// oracle/_ref/librefpipe.so against the Qt stand-ins of oracle/ref_shim/.
//
// TEST INFRASTRUCTURE ONLY: it runs the reference to produce golden vectors
// (tests/golden/make_golden.py) and to check the oracle restatement against
// the reference itself (tests/test_golden.py).  The product never loads it.
//
// The steps follow the reference's own set-up: main.cpp:143-153 (containers,
// formula list) and cRenderJob::Execute, render_job.cpp:393-478 (objects tree,
// sParamRender, sequences, lights, resolution).
#include <cstdio>
#include <cstring>
#include <memory>

#include "formula/definition/all_fractal_list.hpp"
#include "src/calculate_distance.hpp"
#include "src/cimage.hpp"
#include "src/compute_fractal.hpp"
#include "src/fractal_container.hpp"
#include "src/fractparams.hpp"
#include "src/hybrid_fractal_sequences.h"
#include "src/initparameters.hpp"
#include "src/material.h"
#include "src/objects_tree.h"
#include "src/parameters.hpp"
#include "src/primitive_item.h"
#include "src/primitives.h"
#include "src/render_data.hpp"
#include "src/render_worker.hpp"
#include "src/scheduler.hpp"

extern unsigned int gRandomSeed;  // common_math.cpp:47

namespace {

struct Pipeline {
  std::shared_ptr<cParameterContainer> par;
  std::shared_ptr<cFractalContainer> fract;
  std::shared_ptr<sParamRender> params;
  std::shared_ptr<cHybridFractalSequences> fractals;
  std::shared_ptr<sRenderData> data;
  bool prepared = false;
};

void define_formulas() {
  static bool done = false;
  if (!done) {
    DefineFractalList(&newFractalList);  // main.cpp:153
    done = true;
  }
}

}  // namespace

extern "C" {

// Containers holding the reference's defaults (main.cpp:143-150, with the
// first material as render_queue.cpp:70-80 adds it).
void *refp_new(void) {
  define_formulas();
  Pipeline *p = new Pipeline();
  p->par = std::make_shared<cParameterContainer>();
  p->fract = std::make_shared<cFractalContainer>();
  p->par->SetContainerName("main");
  InitParams(p->par);
  InitNodeParams(1, p->par);
  InitMaterialParams(1, p->par);
  InitLightParams(1, p->par);
  for (int i = 0; i < p->fract->size(); i++) {
    p->fract->at(i)->SetContainerName(QString("fractal") + QString::number(i));
    InitFractalParams(p->fract->at(i));
  }
  return p;
}

void refp_free(void *h) { delete static_cast<Pipeline *>(h); }

int refp_prepare(void *h);

// Sets one parameter: fractal < 0 the main container, else fractal slot
// `fractal` (0-based).  kind: 0 int, 1 double, 2 bool, 3 vector (3 doubles).
int refp_set(void *h, int fractal, const char *name, int kind, const double *v) {
  Pipeline *p = static_cast<Pipeline *>(h);
  std::shared_ptr<cParameterContainer> c = fractal < 0 ? p->par : p->fract->at(fractal);
  const QString n(name);
  if (!c->IfExists(n)) return 1;
  switch (kind) {
    case 0: c->Set<int>(n, int(v[0])); break;
    case 1: c->Set<double>(n, v[0]); break;
    case 2: c->Set<bool>(n, v[0] != 0.0); break;
    case 3: c->Set<CVector3>(n, CVector3(v[0], v[1], v[2])); break;
    default: return 2;
  }
  p->prepared = false;
  return 0;
}

// The kind refp_set takes for a parameter of the main container (fractal <
// 0) or of fractal slot `fractal`: 0 int, 1 double, 2 bool, 3 vector; -1 when
// the container has no such parameter or it is of another type.
int refp_param_kind(void *h, int fractal, const char *name) {
  Pipeline *p = static_cast<Pipeline *>(h);
  std::shared_ptr<cParameterContainer> c = fractal < 0 ? p->par : p->fract->at(fractal);
  const QString n(name);
  if (!c->IfExists(n)) return -1;
  switch (c->GetVarType(n)) {
    case parameterContainer::typeInt: return 0;
    case parameterContainer::typeDouble: return 1;
    case parameterContainer::typeBool: return 2;
    case parameterContainer::typeVector3: return 3;
    default: return -1;
  }
}

// Sets a string parameter (node definitions, enumerations by name).
int refp_set_string(void *h, int fractal, const char *name, const char *value) {
  Pipeline *p = static_cast<Pipeline *>(h);
  std::shared_ptr<cParameterContainer> c = fractal < 0 ? p->par : p->fract->at(fractal);
  const QString n(name);
  if (!c->IfExists(n)) return 1;
  c->Set<QString>(n, QString(value));
  p->prepared = false;
  return 0;
}

// Adds the parameters of objects-tree node `id` with their defaults
// (InitNodeParams, initparameters.cpp:2102-2125).
int refp_add_node(void *h, int id) {
  Pipeline *p = static_cast<Pipeline *>(h);
  InitNodeParams(id, p->par);
  p->prepared = false;
  return 0;
}

// Adds the parameters of primitive_<type>_<id> with their defaults
// (InitPrimitiveParams, initparameters.cpp:1313-1420).
int refp_add_primitive(void *h, const char *type_name, int id) {
  Pipeline *p = static_cast<Pipeline *>(h);
  const QString name(type_name);
  const fractal::enumObjectType t = cPrimitives::PrimitiveNameToEnum(name);
  const sPrimitiveItem item(t, id, QString("primitive_%1_%2").arg(name).arg(id), name);
  InitPrimitiveParams(item, p->par);
  p->prepared = false;
  return 0;
}

// The unit direction toward light `index` (0-based) after cLights::Set
// (lights.cpp), as LightShading reads it.
int refp_light_direction(void *h, int index, double *dir) {
  Pipeline *p = static_cast<Pipeline *>(h);
  if (!p->prepared && refp_prepare(h)) return 1;
  if (index < 0 || index >= p->data->lights.GetNumberOfLights()) return 2;
  const cLight *l = p->data->lights.GetLight(index);
  dir[0] = l->lightDirection.x;
  dir[1] = l->lightDirection.y;
  dir[2] = l->lightDirection.z;
  return 0;
}

// cRenderJob::Execute's set-up (render_job.cpp:393-478) for the current
// parameters: objects tree, sParamRender, sequences, lights, materials.
int refp_prepare(void *h) {
  Pipeline *p = static_cast<Pipeline *>(h);
  p->data = std::make_shared<sRenderData>();
  sRenderData &data = *p->data;
  const int width = p->par->Get<int>("image_width"), height = p->par->Get<int>("image_height");
  if (p->par->Get<bool>("legacy_coordinate_system"))
    data.imageRegion.Set(-0.5, -0.5, 0.5, 0.5);
  else
    data.imageRegion.Set(-0.5, 0.5, 0.5, -0.5);
  data.screenRegion.Set(0, 0, width, height);
  CreateMaterialsVector(p->par, &data.materials, false, true, false);
  cObjectsTree tree;
  tree.CreateNodeDataFromParameters(p->par);
  data.nodesDataForRendering = tree.GetNodeDataListForRendering();
  p->params = std::make_shared<sParamRender>(p->par, &data.objectData, &data.nodesDataForRendering, p->fract);
  cObjectsTree tree2;
  tree2.CreateNodeDataFromParameters(p->par);
  std::vector<cObjectsTree::sNodeDataForRendering> nodes = tree2.GetNodeDataListForRendering();
  p->fractals = std::make_shared<cHybridFractalSequences>();
  p->fractals->CreateSequences(p->par, p->fract, nodes);
  if (p->params->objectsTreeEnable) {
    cHybridFractalSequences hs;
    hs.CreateSequences(p->par, p->fract, data.nodesDataForRendering);
    data.hybridFractalSequences = hs;
  }
  data.lights.Set(p->par, p->fract, true, true, false, p->data.get());
  for (const auto &node : data.nodesDataForRendering) {
    if (node.material > 0 && node.internalObjectId >= 0 && node.internalObjectId < int(data.objectData.size()))
      data.objectData[node.internalObjectId].materialId = node.material;
    if (node.internalObjectId >= 0 && node.internalObjectId < int(data.objectData.size())) {
      data.objectData[node.internalObjectId].worldToLocalMatrix = node.worldToLocalMatrix;
      data.objectData[node.internalObjectId].rotationMatrix = node.rotationMatrix;
      data.objectData[node.internalObjectId].repeat = node.repeat;
      data.objectData[node.internalObjectId].absScale = node.absScale;
    }
  }
  data.ValidateObjects();
  p->params->resolution = 1.0 / height;  // render_job.cpp:477
  data.reduceDetail = 1.0;
  // cRenderJob::InitStatistics (render_job.cpp:883-889)
  data.statistics.histogramIterations.Resize(p->par->Get<int>("N"));
  data.statistics.histogramStepCount.Resize(1000);
  data.statistics.Reset();
  p->prepared = true;
  return 0;
}

// CalculateDistance (calculate_distance.cpp:60) at n points.
int refp_distance(void *h, const double *pts, int n, double detail, int normal_mode, double *dist, int *iters) {
  Pipeline *p = static_cast<Pipeline *>(h);
  if (!p->prepared && refp_prepare(h)) return 1;
  for (int i = 0; i < n; i++) {
    sDistanceIn in(CVector3(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]), detail, normal_mode != 0);
    // zero-initialised: the limit-box early-out (calculate_distance.cpp:268-273)
    // returns without setting `iters`
    sDistanceOut out{};
    dist[i] = CalculateDistance(*p->params, *p->fractals, in, &out, p->data.get());
    if (iters) iters[i] = out.iters;
  }
  return 0;
}

// Compute<calcModeNormal> (compute_fractal.cpp:67-654) of the render's
// sequence 0 at n points, as CalculateDistanceSimple calls it
// (calculate_distance.cpp:541-551): z out (3 per point), distance, iters,
// maxiter.
int refp_compute(void *h, const double *pts, int n, int normal_mode, double *z, double *dist, int *iters,
                 int *maxiter) {
  Pipeline *p = static_cast<Pipeline *>(h);
  if (!p->prepared && refp_prepare(h)) return 1;
  const cHybridFractalSequences::sSequence *seq = p->data->hybridFractalSequences.GetSequence(0);
  if (!seq) return 2;
  const sParamRender &params = *p->params;
  const int maxiterMultiplier = (normal_mode && params.common.iterThreshMode) ? 5 : 1;
  for (int i = 0; i < n; i++) {
    sFractalIn fin(CVector3(pts[3 * i], pts[3 * i + 1], pts[3 * i + 2]), params.minN, -1, maxiterMultiplier, 0,
                   &params.common, -1, normal_mode != 0);
    sFractalOut fout;
    fout.colorIndex = 0;
    Compute<fractal::calcModeNormal>(seq, fin, &fout);
    z[3 * i] = fout.z.x;
    z[3 * i + 1] = fout.z.y;
    z[3 * i + 2] = fout.z.z;
    dist[i] = fout.distance;
    iters[i] = fout.iters;
    maxiter[i] = fout.maxiter ? 1 : 0;
  }
  return 0;
}

// The render's sequence 0: table (up to `cap` entries), length, DE function
// type, DE type, analytic DE function, per-slot bailout.
int refp_sequence(void *h, int *seq_out, int cap, int *length, int *de_function, int *de_type, int *analytic,
                  double *bailout, int *n_slots) {
  Pipeline *p = static_cast<Pipeline *>(h);
  if (!p->prepared && refp_prepare(h)) return 1;
  const cHybridFractalSequences::sSequence *seq = p->data->hybridFractalSequences.GetSequence(0);
  if (!seq) return 2;
  *length = seq->length;
  for (int i = 0; i < seq->length && i < cap; i++) seq_out[i] = seq->seqence[i];
  *de_function = int(seq->DEFunctionType);
  *de_type = int(seq->DEType);
  *analytic = int(seq->DEAnalyticFunction);
  *n_slots = int(seq->fractData.size());
  for (size_t i = 0; i < seq->fractData.size() && i < 9; i++) bailout[i] = seq->fractData[i].bailout;
  return 0;
}

// One frame by cRenderWorker::doWork on this thread (one worker, no
// progressive passes: lines in order, pixels left to right), with the
// process-global Park-Miller seed set to `seed` just before the pixel loop
// (the march jitter draws one number per march step).  Outputs, W x H each:
// zbuffer (float depth, 1e20 on miss), world normal (3 floats, only when
// normal_world != NULL), the shadows channel (3 floats, when shadows !=
// NULL) and the 8-bit image (3 bytes, when rgb8 != NULL).
int refp_render(void *h, unsigned int seed, float *zbuf, float *normal_world, float *shadows,
                unsigned char *rgb8) {
  Pipeline *p = static_cast<Pipeline *>(h);
  if (refp_prepare(h)) return 1;
  const int width = p->par->Get<int>("image_width"), height = p->par->Get<int>("image_height");
  std::shared_ptr<cImage> image = std::make_shared<cImage>(width, height);
  sImageOptional opt;
  opt.optionalNormalWorld = normal_world != nullptr;
  opt.optionalShadows = shadows != nullptr;
  image->ChangeSize(width, height, opt);  // allocates the optional channels
  auto scheduler = std::make_shared<cScheduler>(p->data->screenRegion, 1);
  auto td = std::make_shared<cRenderWorker::sThreadData>();
  td->id = 1;
  td->startLine = 0;
  td->scheduler = scheduler;
  bool stop = false;
  p->data->stopRequest = &stop;
  {
    cRenderWorker worker(p->params, p->fractals, td, p->data, image);
    gRandomSeed = seed;
    worker.doWork();
  }
  image->CompileImage();
  const quint8 *img8 = image->ConvertTo8bitChar();
  for (int y = 0; y < height; y++)
    for (int x = 0; x < width; x++) {
      const int i = y * width + x;
      if (zbuf) zbuf[i] = image->GetPixelZBuffer(x, y);
      if (normal_world) {
        const sRGBFloat nw = image->GetPixelNormalWorld(x, y);
        normal_world[3 * i] = nw.R;
        normal_world[3 * i + 1] = nw.G;
        normal_world[3 * i + 2] = nw.B;
      }
      if (shadows) {
        const sRGBFloat s = image->GetPixelShadows(x, y);
        shadows[3 * i] = s.R;
        shadows[3 * i + 1] = s.G;
        shadows[3 * i + 2] = s.B;
      }
      if (rgb8 && img8)
        for (int k = 0; k < 3; k++) rgb8[3 * i + k] = img8[3 * i + k];
    }
  return 0;
}

}  // extern "C"
