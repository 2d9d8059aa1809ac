// ref_pipeline_stubs.cpp - stand-ins for the definitions that the reference's
// hot-path sources link against but whose own sources need Qt's GUI, file,
// network or image classes (or GSL): logging, texture loading, the random
// generator of the random lights, the netrender and system globals, and the
// Qt signals that moc would generate.  The distance-estimation path of the
// harness (oracle/ref_pipeline.cpp) holds these objects but, with textures,
// random lights and netrender off, calls none of them except the logging and
// the signals, which do nothing here.  TEST INFRASTRUCTURE ONLY.
#include "src/lights.hpp"
#include "src/netrender.hpp"
#include "src/random.hpp"
#include "src/render_worker.hpp"
#include "src/system.hpp"
#include "src/system_data.hpp"
#include "src/system_directories.hpp"
#include "src/texture.hpp"
#include "src/write_log.hpp"

void WriteLog(const QString &, int) {}
void WriteLogCout(const QString &, int) {}
void WriteLogString(const QString &, const QString &, int) {}
void WriteLogDouble(const QString &, double, int) {}
void WriteLogInt(const QString &, int, int) {}
void WriteLogSizeT(const QString &, size_t, int) {}

cTexture::cTexture() {}
cTexture::cTexture(QString, enumUseMipmaps, int, bool, bool) {}
cTexture::cTexture(const cTexture &) {}
cTexture::cTexture(cTexture &&) {}
cTexture &cTexture::operator=(cTexture &&) { return *this; }
cTexture &cTexture::operator=(const cTexture &) { return *this; }
sRGBFloat cTexture::Pixel(CVector2<float>, float) const { return sRGBFloat(); }
sRGBFloat cTexture::Pixel(float, float, float) const { return sRGBFloat(); }
CVector3 cTexture::NormalMapFromBumpMap(CVector2<float>, float, float) const { return CVector3(0.0, 0.0, 1.0); }
CVector3 cTexture::NormalMap(CVector2<float>, float, bool, float) const { return CVector3(0.0, 0.0, 1.0); }

cRandom::cRandom() : gBaseRand(nullptr) {}
cRandom::~cRandom() {}
void cRandom::Initialize(int) const {}
int cRandom::Random(unsigned long) const { return 0; }
double cRandom::Random(double min, double, double) const { return min; }
double cRandom::DoubleRandom(double min, double) const { return min; }

cNetRender *gNetRender = nullptr;
sSystem systemData;
sSystemDirectories systemDirectories;
int get_cpu_count() { return 1; }
QString sSystemDirectories::GetDataDirectoryUsed() const { return QString("."); }

// Qt signals (moc output in the reference's build)
void cRenderWorker::finished() {}
void cRenderWorker::error(const QString &) {}
void cLights::updateProgressAndStatus(const QString &, const QString &, double) {}
