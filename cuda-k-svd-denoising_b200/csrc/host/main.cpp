// Command-line driver (src/main.cpp:114-124): runs every image of a
// config.json through the sm_100a denoiser and prints the reference's
// per-image timing / PSNR report.
#include <cstdio>

extern "C" int ksvd_run_batch(const char* json_path, int verbose);

int main(int argc, char* argv[]) {
  const char* file = "../config.json";
  if (argc == 2) file = argv[1];
  const int failures = ksvd_run_batch(file, 1);
  return failures < 0 ? 2 : (failures > 0 ? 1 : 0);
}
