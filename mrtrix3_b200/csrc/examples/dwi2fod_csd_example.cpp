// dwi2fod_csd_example: the csd branch of MRtrix3's cmd/dwi2fod.cpp:256-281
// written against the drop-in CSD surface (csd.hpp), on raw files:
//
//   dwi2fod_csd_example grad.txt response.txt dwi.f32 n_voxels fod.f32
//                       [-mask mask.u8] [-lmax L] [-niter N] [-per_voxel K]
//
// grad.txt: one "x y z b" row per volume; response.txt: zonal SH
// coefficients; dwi.f32: n_voxels x n_volumes float32, voxel-interleaved;
// fod.f32: n_voxels x nSH float32.  -per_voxel K additionally runs the
// per-voxel set()/iterate()/FOD() loop (CSD_Processor, dwi2fod.cpp:128-147)
// on the first K voxels and reports the largest difference to the batch.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "../csd.hpp"

using MR::DWI::SDeconv::CSD;
using MR::DWI::SDeconv::CSDOptions;

static std::vector<double> read_table(const std::string& path) {
  std::ifstream f(path);
  if (!f) throw MR::DWI::SDeconv::Exception("cannot open " + path);
  std::vector<double> v;
  double x;
  while (f >> x) v.push_back(x);
  return v;
}

int main(int argc, char** argv) {
  if (argc < 6) {
    std::fprintf(stderr, "usage: %s grad.txt response.txt dwi.f32 n_voxels fod.f32 [-mask m.u8] [-lmax L] "
                         "[-niter N] [-per_voxel K]\n", argv[0]);
    return 2;
  }
  try {
    const std::vector<double> grad = read_table(argv[1]);
    const int64_t nvox = std::atoll(argv[4]);
    CSDOptions opt;
    std::string mask_path;
    int per_voxel = 0;
    for (int i = 6; i + 1 < argc; i += 2) {
      const std::string o = argv[i];
      if (o == "-mask") mask_path = argv[i + 1];
      else if (o == "-lmax") opt.lmax = {uint32_t(std::atoi(argv[i + 1]))};
      else if (o == "-niter") { opt.niter = size_t(std::atoi(argv[i + 1])); opt.has_niter = true; }
      else if (o == "-per_voxel") per_voxel = std::atoi(argv[i + 1]);
      else throw MR::DWI::SDeconv::Exception("unknown option " + o);
    }
    // dwi2fod.cpp:262-271
    CSD::Shared shared(grad);
    shared.parse_cmdline_options(opt);
    shared.set_response(std::string(argv[2]));
    shared.init();
    const size_t nvol = grad.size() / 4, nsh = shared.nSH();
    std::vector<float> dwi(size_t(nvox) * nvol), fod(size_t(nvox) * nsh);
    std::ifstream fi(argv[3], std::ios::binary);
    fi.read(reinterpret_cast<char*>(dwi.data()), std::streamsize(dwi.size() * sizeof(float)));
    if (!fi) throw MR::DWI::SDeconv::Exception("short read on dwi file");
    std::vector<uint8_t> mask;
    if (!mask_path.empty()) {
      mask.resize(size_t(nvox));
      std::ifstream fm(mask_path, std::ios::binary);
      fm.read(reinterpret_cast<char*>(mask.data()), std::streamsize(mask.size()));
    }
    // dwi2fod.cpp:275-281: the whole volume in one batched call
    MR::DWI::SDeconv::dwi2fod_csd(shared, dwi.data(), nvox, mask.empty() ? nullptr : mask.data(), fod.data());
    std::ofstream fo(argv[5], std::ios::binary);
    fo.write(reinterpret_cast<const char*>(fod.data()), std::streamsize(fod.size() * sizeof(float)));
    // CSD_Processor::operator() per voxel (dwi2fod.cpp:128-147)
    double worst = 0.0;
    CSD sdeconv(shared);
    for (int v = 0; v < per_voxel && v < nvox; ++v) {
      std::vector<double> data(shared.dwis.size());
      for (size_t n = 0; n < shared.dwis.size(); ++n) {
        data[n] = dwi[size_t(v) * nvol + shared.dwis[n]];
        if (data[n] < 0.0) data[n] = 0.0;
      }
      sdeconv.set(data);
      for (size_t n = 0; n < shared.niter; ++n)
        if (sdeconv.iterate()) break;
      const std::vector<double>& F = sdeconv.FOD();
      double mx = 0.0, d = 0.0;
      for (size_t c = 0; c < nsh; ++c) {
        mx = std::max(mx, std::fabs(double(fod[size_t(v) * nsh + c])));
        d = std::max(d, std::fabs(F[c] - double(fod[size_t(v) * nsh + c])));
      }
      worst = std::max(worst, mx > 0 ? d / mx : d);
    }
    std::printf("nSH %zu voxels %lld per_voxel_max_rel_diff %.3e\n", nsh, (long long)nvox, worst);
  } catch (const std::exception& e) {
    std::fprintf(stderr, "dwi2fod_csd_example: %s\n", e.what());
    return 1;
  }
  return 0;
}
