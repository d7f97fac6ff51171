// C++ host interface mirroring the reference's denoisingLib
// (src/lib/denoisingLib/denoisingLib.h): DenoiserType and its string map,
// Denoiser::factory, denoising() with status 0 / -1 / -2 / -3,
// getTimeElapsed(), getPsnr(), BatchDenoiser::factory(config.json).
// Every computation goes through the C ABI in include/ksvd_sm100.h.
#pragma once

#include <cstdint>
#include <map>
#include <string>
#include <vector>

#include "ksvd_sm100.h"

namespace denoising {

class Denoiser;
class Sm100KSvdDenoiser;
class BatchDenoiser;

// denoisingLib.h:21; CUDA_K_SM100A is the sm_100a engine (the other three
// names are accepted and run it too).
enum DenoiserType { CUDA_K_GESVD, CUDA_K_GESVDJ, CUDA_K_GESVDA, CUDA_K_SM100A };

// denoisingLib.h:23-31
struct DenoiserTypeMap : public std::map<std::string, DenoiserType> {
  DenoiserTypeMap() {
    (*this)["CUDA_K_GESVD"] = CUDA_K_GESVD;
    (*this)["CUDA_K_GESVDJ"] = CUDA_K_GESVDJ;
    (*this)["CUDA_K_GESVDA"] = CUDA_K_GESVDA;
    (*this)["CUDA_K_SM100A"] = CUDA_K_SM100A;
  }
};

// baseUtilityLib.h:38-44 (milliseconds)
struct TimeElapsed {
  int64_t init = 0, working = 0, finalize = 0;
  int64_t getTotalTime() const { return init + working + finalize; }
};

// A float image, row-major (height x width).
struct Image {
  int width = 0, height = 0;
  std::vector<float> data;
};

// PGM (P2/P5) and PPM (P3/P6), 8 or 16 bit.  Colour images are kept as three
// planes (R, G, B) concatenated in `data` with *channels = 3.
bool read_pnm(const std::string& path, Image* img, int* channels, std::string* err);
// Writes an 8-bit PGM; values are clamped to [0, 255] and rounded.
bool write_pgm(const std::string& path, const Image& img, std::string* err);
// Luma of an RGB image, ITU-R BT.601 studio range: Y = 16 + (65.481 R +
// 128.553 G + 24.966 B) / 255 (the reference takes channel 0 of CImg's
// RGBtoYCbCr, denoiser.cpp:47-48).
Image rgb_to_luma(const Image& rgb3);
// Noise variance estimate from the Laplacian-like 3x3 mask (Immerkaer,
// "Fast noise variance estimation", 1996).  The reference calls CImg's
// variance_noise() (denoiser.cpp:56), a third-party routine not available
// here; config key "noiseVariance" overrides this estimate.
double estimate_noise_variance(const Image& img);
// 10 log10(255^2 / MSE) (CImg::PSNR with its default 255 peak)
double psnr(const Image& a, const Image& b);
// Min-max normalisation to [0, 255] (denoiser.cpp:75)
Image normalize_0_255(const Image& img);

class Denoiser {
 public:
  virtual ~Denoiser();
  // denoiser.cpp:108-127
  static Denoiser* factory(DenoiserType type, const std::string& inputFile, const std::string& outputFile);
  // 0 done, -1 image loading failed, -2 denoising failed, -3 image saving failed
  virtual signed char denoising() = 0;
  TimeElapsed* getTimeElapsed();
  // {PSNR before, PSNR after}; -1 when no reference image was given
  std::vector<double>* getPsnr();

  // parameters (denoisingLib.h:44-56), set by BatchDenoiser::factory
  int patchWidthDim = 8;
  int patchHeightDim = 8;
  int slidingWidth = 2;
  int slidingHeight = 2;
  int subImageWidthDim = 0;
  int subImageHeightDim = 0;
  int ompIter = 5;
  int atoms = 256;
  int iter = 10;
  int minOmpIterBatch = 0;
  float sigma = 0.0f;          // noise variance, from noiseVariance or the estimate
  double noiseVariance = -1.0; // config override (not a reference key)
  bool speckle = false;
  bool bw = true;
  int precision = KSVD_PREC_FP32;
  unsigned compat = KSVD_COMPAT_REFERENCE;
  std::string refImage;
  std::string lastError;

 protected:
  Denoiser();
  virtual bool loadImage();
  virtual bool saveImage();
  virtual bool internalDenoising() = 0;

  std::string inputFile, outputFile;
  DenoiserType type = CUDA_K_SM100A;
  Image input, output;
  TimeElapsed timeElapsed;
  std::vector<double> psnrv{-1.0, -1.0};

  friend class BatchDenoiser;
};

class Sm100KSvdDenoiser : public Denoiser {
 public:
  ~Sm100KSvdDenoiser() override;
  signed char denoising() override;
  const ksvd_stats& stats() const { return stats_; }

 protected:
  bool internalDenoising() override;

 private:
  Sm100KSvdDenoiser() = default;
  ksvd_stats stats_{};
  friend class Denoiser;
};

class BatchDenoiser {
 public:
  ~BatchDenoiser();
  std::vector<Denoiser*> getDenoiserList();
  // batch_denoiser.cpp:36-118; returns nullptr (and sets *err) on a bad file
  static BatchDenoiser* factory(const std::string& jsonFile, std::string* err = nullptr);

 protected:
  std::vector<Denoiser*> denoisers;

 private:
  BatchDenoiser() = default;
};

}  // namespace denoising
