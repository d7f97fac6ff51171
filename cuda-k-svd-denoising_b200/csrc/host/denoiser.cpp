// C++ host mirror of the reference's denoisingLib (denoiser.cpp,
// cuda_svd_denoiser.cu:86-120, batch_denoiser.cpp) on top of the C ABI.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <sstream>

#include "denoising_lib.h"
#include "json_lite.h"

namespace denoising {

using clk = std::chrono::steady_clock;

static int64_t ms_between(clk::time_point a, clk::time_point b) {
  return int64_t(std::chrono::duration_cast<std::chrono::milliseconds>(b - a).count());
}

// ---------------------------------------------------------------------------
// Image I/O and helpers
// ---------------------------------------------------------------------------
static bool pnm_token(std::istream& in, std::string* tok) {
  tok->clear();
  int c;
  while ((c = in.get()) != EOF) {
    if (c == '#') {
      while ((c = in.get()) != EOF && c != '\n') {
      }
      continue;
    }
    if (!std::isspace(c)) {
      tok->push_back(char(c));
      break;
    }
  }
  while ((c = in.peek()) != EOF && !std::isspace(c) && c != '#') tok->push_back(char(in.get()));
  return !tok->empty();
}

bool read_pnm(const std::string& path, Image* img, int* channels, std::string* err) {
  std::ifstream in(path, std::ios::binary);
  if (!in) {
    *err = "cannot open " + path;
    return false;
  }
  std::string magic, ws, hs, ms;
  if (!pnm_token(in, &magic) || !pnm_token(in, &ws) || !pnm_token(in, &hs) || !pnm_token(in, &ms)) {
    *err = "bad PNM header in " + path;
    return false;
  }
  const bool ascii = magic == "P2" || magic == "P3";
  const int ch = (magic == "P3" || magic == "P6") ? 3 : (magic == "P2" || magic == "P5") ? 1 : 0;
  if (!ch) {
    *err = "unsupported PNM type " + magic;
    return false;
  }
  const int W = std::atoi(ws.c_str()), H = std::atoi(hs.c_str()), maxv = std::atoi(ms.c_str());
  if (W <= 0 || H <= 0 || maxv <= 0 || maxv > 65535) {
    *err = "bad PNM dimensions";
    return false;
  }
  img->width = W;
  img->height = H;
  img->data.assign(size_t(W) * H * ch, 0.0f);
  const size_t plane = size_t(W) * H;
  if (!ascii) in.get();  // single whitespace after maxval
  for (size_t px = 0; px < plane; ++px) {
    for (int c = 0; c < ch; ++c) {
      unsigned v = 0;
      if (ascii) {
        std::string t;
        if (!pnm_token(in, &t)) {
          *err = "truncated PNM data";
          return false;
        }
        v = unsigned(std::atoi(t.c_str()));
      } else if (maxv < 256) {
        int b = in.get();
        if (b == EOF) {
          *err = "truncated PNM data";
          return false;
        }
        v = unsigned(b);
      } else {
        int hi = in.get(), lo = in.get();
        if (lo == EOF) {
          *err = "truncated PNM data";
          return false;
        }
        v = unsigned(hi) << 8 | unsigned(lo);
      }
      img->data[size_t(c) * plane + px] = float(v);  // planar, like CImg
    }
  }
  *channels = ch;
  return true;
}

bool write_pgm(const std::string& path, const Image& img, std::string* err) {
  std::ofstream out(path, std::ios::binary);
  if (!out) {
    *err = "cannot write " + path;
    return false;
  }
  out << "P5\n" << img.width << " " << img.height << "\n255\n";
  std::vector<unsigned char> row(size_t(img.width) * img.height);
  for (size_t i = 0; i < row.size(); ++i) {
    float v = std::round(img.data[i]);
    row[i] = (unsigned char)(v < 0.0f ? 0.0f : (v > 255.0f ? 255.0f : v));
  }
  out.write(reinterpret_cast<const char*>(row.data()), std::streamsize(row.size()));
  if (!out) {
    *err = "write failed for " + path;
    return false;
  }
  return true;
}

Image rgb_to_luma(const Image& rgb3) {
  Image y;
  y.width = rgb3.width;
  y.height = rgb3.height;
  const size_t plane = size_t(rgb3.width) * rgb3.height;
  y.data.resize(plane);
  for (size_t i = 0; i < plane; ++i) {
    const float r = rgb3.data[i], g = rgb3.data[plane + i], b = rgb3.data[2 * plane + i];
    y.data[i] = 16.0f + (65.481f * r + 128.553f * g + 24.966f * b) / 255.0f;
  }
  return y;
}

double estimate_noise_variance(const Image& img) {
  const int W = img.width, H = img.height;
  if (W < 3 || H < 3) return 0.0;
  double acc = 0.0;
  for (int y = 1; y + 1 < H; ++y)
    for (int x = 1; x + 1 < W; ++x) {
      auto at = [&](int dx, int dy) { return double(img.data[size_t(y + dy) * W + (x + dx)]); };
      const double v = at(-1, -1) - 2 * at(0, -1) + at(1, -1) - 2 * at(-1, 0) + 4 * at(0, 0) - 2 * at(1, 0) +
                       at(-1, 1) - 2 * at(0, 1) + at(1, 1);
      acc += std::fabs(v);
    }
  const double pi = 3.14159265358979323846;
  const double sigma = std::sqrt(pi / 2.0) * acc / (6.0 * double(W - 2) * double(H - 2));
  return sigma * sigma;
}

double psnr(const Image& a, const Image& b) {
  const size_t n = std::min(a.data.size(), b.data.size());
  if (n == 0) return -1.0;
  double mse = 0.0;
  for (size_t i = 0; i < n; ++i) {
    const double d = double(a.data[i]) - double(b.data[i]);
    mse += d * d;
  }
  mse /= double(n);
  if (mse == 0.0) return INFINITY;
  return 10.0 * std::log10(255.0 * 255.0 / mse);
}

Image normalize_0_255(const Image& img) {
  Image o = img;
  if (img.data.empty()) return o;
  const auto mm = std::minmax_element(img.data.begin(), img.data.end());
  const float lo = *mm.first, hi = *mm.second;
  const float sc = (hi > lo) ? 255.0f / (hi - lo) : 0.0f;
  for (auto& v : o.data) v = (v - lo) * sc;
  return o;
}

// ---------------------------------------------------------------------------
// Denoiser (denoiser.cpp)
// ---------------------------------------------------------------------------
Denoiser::Denoiser() = default;
Denoiser::~Denoiser() = default;

Denoiser* Denoiser::factory(DenoiserType type, const std::string& inputFile, const std::string& outputFile) {
  Denoiser* d = nullptr;
  switch (type) {
    case CUDA_K_GESVD:
    case CUDA_K_GESVDJ:
    case CUDA_K_GESVDA:
    case CUDA_K_SM100A:
      d = new Sm100KSvdDenoiser();
      break;
    default:
      return nullptr;
  }
  d->type = type;
  d->inputFile = inputFile;
  d->outputFile = outputFile;
  return d;
}

TimeElapsed* Denoiser::getTimeElapsed() { return &timeElapsed; }
std::vector<double>* Denoiser::getPsnr() { return &psnrv; }

// denoiser.cpp:37-62: read, luma for colour input when B&W is false (the
// first channel otherwise, as CImg's planar data() gives), noise variance.
bool Denoiser::loadImage() {
  const auto t0 = clk::now();
  Image raw;
  int ch = 0;
  if (!read_pnm(inputFile, &raw, &ch, &lastError)) return false;
  if (ch == 3 && !bw) {
    input = rgb_to_luma(raw);
  } else {
    input.width = raw.width;
    input.height = raw.height;
    input.data.assign(raw.data.begin(), raw.data.begin() + size_t(raw.width) * raw.height);
  }
  sigma = float(noiseVariance > 0.0 ? noiseVariance : estimate_noise_variance(input));
  timeElapsed.init = ms_between(t0, clk::now());
  return true;
}

// denoiser.cpp:68-99: min-max normalise, save, PSNR against the reference
// image when one is given (refImage ending in '/' means none).
bool Denoiser::saveImage() {
  const auto t0 = clk::now();
  Image norm = normalize_0_255(output);
  if (!write_pgm(outputFile, norm, &lastError)) return false;
  timeElapsed.finalize = ms_between(t0, clk::now());
  if (refImage.empty() || refImage.back() == '/') {
    psnrv = {-1.0, -1.0};
    return true;
  }
  Image ref, old;
  int c1 = 0, c2 = 0;
  if (!read_pnm(refImage, &ref, &c1, &lastError) || !read_pnm(inputFile, &old, &c2, &lastError)) {
    psnrv = {-1.0, -1.0};
    return true;
  }
  psnrv = {psnr(ref, old), psnr(ref, norm)};
  return true;
}

// ---------------------------------------------------------------------------
// Sm100KSvdDenoiser (CudaKSvdDenoiser, cuda_svd_denoiser.cu:86-216)
// ---------------------------------------------------------------------------
Sm100KSvdDenoiser::~Sm100KSvdDenoiser() = default;

signed char Sm100KSvdDenoiser::denoising() {
  if (!loadImage()) return -1;
  if (!internalDenoising()) return -2;
  if (!saveImage()) return -3;
  return 0;
}

bool Sm100KSvdDenoiser::internalDenoising() {
  const auto t0 = clk::now();
  ksvd_params p;
  ksvd_params_default(&p);
  p.patch_width_dim = patchWidthDim;
  p.patch_height_dim = patchHeightDim;
  p.sliding_width = slidingWidth;
  p.sliding_height = slidingHeight;
  p.atoms = atoms;
  p.ksvd_iter = iter;
  p.omp_iter = ompIter;
  p.bw = bw ? 1 : 0;
  p.speckle = speckle ? 1 : 0;
  p.type = int(type);
  p.min_omp_iter_batch = minOmpIterBatch;
  p.sub_image_width_dim = subImageWidthDim;
  p.sub_image_height_dim = subImageHeightDim;
  p.precision = precision;
  p.compat = compat;
  ksvd_ctx* ctx = nullptr;
  ksvd_status st = ksvd_create(&p, &ctx);
  if (st != KSVD_OK) {
    lastError = std::string("ksvd_create: ") + ksvd_status_string(st);
    return false;
  }
  // The reference transposes the loaded image and hands its column-major
  // matrix on (denoiser.cpp:46-51); its patch walk, dictionary seeds and
  // sub-images therefore follow the image's columns.  The library gets the
  // same buffer, this image transposed as a row-major image, and the result
  // is transposed back.
  const int W = input.width, H = input.height;
  std::vector<float> tin(size_t(W) * H), tout(size_t(W) * H, 0.0f);
  for (int y = 0; y < H; ++y)
    for (int x = 0; x < W; ++x) tin[size_t(x) * H + y] = input.data[size_t(y) * W + x];
  st = ksvd_denoise(ctx, tin.data(), H, W, sigma, tout.data(), &stats_);
  if (st != KSVD_OK) lastError = ksvd_last_error(ctx);
  output.width = W;
  output.height = H;
  output.data.assign(size_t(W) * H, 0.0f);
  for (int y = 0; y < H; ++y)
    for (int x = 0; x < W; ++x) output.data[size_t(y) * W + x] = tout[size_t(x) * H + y];
  ksvd_destroy(ctx);
  timeElapsed.working = ms_between(t0, clk::now());
  return st == KSVD_OK;
}

// ---------------------------------------------------------------------------
// BatchDenoiser (batch_denoiser.cpp:36-118)
// ---------------------------------------------------------------------------
BatchDenoiser::~BatchDenoiser() {
  for (Denoiser* d : denoisers) delete d;
}

std::vector<Denoiser*> BatchDenoiser::getDenoiserList() { return denoisers; }

static int precision_from(const ksvd_json::Value& v, const std::string& key, int dflt) {
  const ksvd_json::Value* x = v.get(key);
  if (!x) return dflt;
  if (x->kind == ksvd_json::Value::Number) return int(x->num);
  if (x->kind == ksvd_json::Value::String) {
    if (x->str == "FP32") return KSVD_PREC_FP32;
    if (x->str == "BF16") return KSVD_PREC_BF16_RESCORE;
    if (x->str == "FP16") return KSVD_PREC_FP16_RESCORE;
  }
  return dflt;
}

BatchDenoiser* BatchDenoiser::factory(const std::string& jsonFile, std::string* err) {
  ksvd_json::Value config;
  std::string e;
  if (!ksvd_json::parse_file(jsonFile, &config, &e) || config.kind != ksvd_json::Value::Object) {
    if (err) *err = e.empty() ? "config is not a JSON object" : e;
    return nullptr;
  }
  static const ksvd_json::Value empty;
  const ksvd_json::Value* gp = config.get("globalParams");
  const ksvd_json::Value& g = gp ? *gp : empty;
  const std::string inputFolder = config.string("inputFolder", "");
  const std::string outputFolder = config.string("outputFolder", "");
  const ksvd_json::Value* files = config.get("files");

  // globals (batch_denoiser.cpp:60-73); defaults of denoisingLib.h:44-56 when absent
  const int gPW = int(g.number("patchWidthDim", 8)), gPH = int(g.number("patchHeightDim", 8));
  const int gSW = int(g.number("slidingWidth", 2)), gSH = int(g.number("slidingHeight", 2));
  const bool gSpeckle = g.boolean("speckle", false), gBW = g.boolean("B&W", true);
  const std::string gType = g.string("type", "CUDA_K_SM100A");
  const int gAtoms = int(g.number("atoms", 256)), gIter = int(g.number("ksvdIter", 10));
  const int gOmp = int(g.number("ompIter", 5)), gMinOmp = int(g.number("minOmpIterBatch", 0));
  const int gSubW = int(g.number("subImageWidthDim", 0)), gSubH = int(g.number("subImageHeightDim", 0));
  const double gNoise = g.number("noiseVariance", -1.0);
  const int gPrec = precision_from(g, "precision", KSVD_PREC_FP32);
  const unsigned gCompat = unsigned(g.number("compat", double(KSVD_COMPAT_REFERENCE)));

  DenoiserTypeMap map;
  auto* batch = new BatchDenoiser();
  if (files && files->kind == ksvd_json::Value::Array) {
    for (const ksvd_json::Value& f : files->arr) {
      const int pw = int(f.number("patchWidthDim", gPW)), ph = int(f.number("patchHeightDim", gPH));
      const std::string name = f.string("name", "");
      const std::string type = f.string("type", gType);
      // std::map::operator[] on an unknown name yields CUDA_K_GESVD, as in the reference
      Denoiser* d = Denoiser::factory(map[type], inputFolder + "/" + name,
                                      outputFolder + "/" + std::to_string(pw) + "_" + std::to_string(ph) + "_" + name);
      d->patchWidthDim = pw;
      d->patchHeightDim = ph;
      d->slidingWidth = int(f.number("slidingWidth", gSW));
      d->slidingHeight = int(f.number("slidingHeight", gSH));
      d->refImage = inputFolder + "/" + f.string("ref", "");
      d->ompIter = int(f.number("ompIter", gOmp));
      d->atoms = int(f.number("atoms", gAtoms));
      d->iter = int(f.number("ksvdIter", gIter));
      d->speckle = f.boolean("speckle", gSpeckle);
      d->bw = f.boolean("B&W", gBW);
      d->minOmpIterBatch = int(f.number("minOmpIterBatch", gMinOmp));
      d->subImageWidthDim = int(f.number("subImageWidthDim", gSubW));
      d->subImageHeightDim = int(f.number("subImageHeightDim", gSubH));
      d->noiseVariance = f.number("noiseVariance", gNoise);
      d->precision = precision_from(f, "precision", gPrec);
      d->compat = unsigned(f.number("compat", double(gCompat)));
      batch->denoisers.push_back(d);
    }
  }
  return batch;
}

}  // namespace denoising

// ---------------------------------------------------------------------------
// C ABI over the config reader (for callers outside C++)
// ---------------------------------------------------------------------------
using denoising::BatchDenoiser;
using denoising::Denoiser;

static void copy_str(char* dst, size_t cap, const std::string& s) {
  if (!dst || cap == 0) return;
  const size_t n = std::min(cap - 1, s.size());
  std::memcpy(dst, s.data(), n);
  dst[n] = '\0';
}

extern "C" int ksvd_batch_count(const char* json_path) {
  if (!json_path) return -1;
  BatchDenoiser* b = BatchDenoiser::factory(json_path);
  if (!b) return -1;
  const int n = int(b->getDenoiserList().size());
  delete b;
  return n;
}

extern "C" ksvd_status ksvd_batch_entry(const char* json_path, int index, ksvd_params* p, char* input_path,
                                        char* output_path, char* ref_path, size_t cap, double* noise_variance) {
  if (!json_path || !p) return KSVD_ERR_INVALID;
  BatchDenoiser* b = BatchDenoiser::factory(json_path);
  if (!b) return KSVD_ERR_INVALID;
  auto list = b->getDenoiserList();
  if (index < 0 || index >= int(list.size())) {
    delete b;
    return KSVD_ERR_INVALID;
  }
  struct Peek : public Denoiser {
    static void fill(Denoiser* d, ksvd_params* p, char* in, char* out, char* ref, size_t cap, double* nv) {
      Peek* x = static_cast<Peek*>(d);
      ksvd_params_default(p);
      p->patch_width_dim = x->patchWidthDim;
      p->patch_height_dim = x->patchHeightDim;
      p->sliding_width = x->slidingWidth;
      p->sliding_height = x->slidingHeight;
      p->atoms = x->atoms;
      p->ksvd_iter = x->iter;
      p->omp_iter = x->ompIter;
      p->bw = x->bw ? 1 : 0;
      p->speckle = x->speckle ? 1 : 0;
      p->type = int(x->type);
      p->min_omp_iter_batch = x->minOmpIterBatch;
      p->sub_image_width_dim = x->subImageWidthDim;
      p->sub_image_height_dim = x->subImageHeightDim;
      p->precision = x->precision;
      p->compat = x->compat;
      copy_str(in, cap, x->inputFile);
      copy_str(out, cap, x->outputFile);
      copy_str(ref, cap, x->refImage);
      if (nv) *nv = x->noiseVariance;
    }
  };
  Peek::fill(list[size_t(index)], p, input_path, output_path, ref_path, cap, noise_variance);
  delete b;
  return KSVD_OK;
}

extern "C" int ksvd_run_batch(const char* json_path, int verbose) {
  if (!json_path) return -1;
  std::string err;
  BatchDenoiser* b = BatchDenoiser::factory(json_path, &err);
  if (!b) {
    if (verbose) std::fprintf(stderr, "config: %s\n", err.c_str());
    return -1;
  }
  int failures = 0;
  double init = 0, work = 0, fin = 0;
  auto list = b->getDenoiserList();
  for (size_t i = 0; i < list.size(); ++i) {
    Denoiser* d = list[i];
    const signed char st = d->denoising();
    if (st == 0) {
      const auto* t = d->getTimeElapsed();
      init += double(t->init);
      work += double(t->working);
      fin += double(t->finalize);
      if (verbose) {
        std::printf("\n## Image: %zu execution time: %.3f s\n", i + 1, double(t->getTotalTime()) / 1000.0);
        std::printf("    init time: %lld ms\n    working time: %.3f s\n    finalize time: %lld ms\n",
                    (long long)t->init, double(t->working) / 1000.0, (long long)t->finalize);
        const auto* ps = d->getPsnr();
        if ((*ps)[0] >= 0) std::printf("    PSNR before:%g\n    PSNR after:%g\n", (*ps)[0], (*ps)[1]);
      }
    } else {
      ++failures;
      if (verbose) {
        const char* what = st == -1 ? "Image Loading Failed" : st == -2 ? "Denoising Failed" : "Image Saving Failed";
        std::printf("%s (%s)\n", what, d->lastError.c_str());
      }
    }
  }
  if (verbose) {
    std::printf("\n# Total Batch execution time: %g s\n", (init + fin + work) / 1000.0);
    std::printf("    Total Batch init time: %g s\n    Total Batch working time: %g s\n", init / 1000.0, work / 1000.0);
    std::printf("    Total Batch finalize time: %g s\n", fin / 1000.0);
  }
  delete b;
  return failures;
}
