// piks3d — command-line host of the B200 solver, following PIKS3D's `program main`
// (main.F90:52-147) for one process: reads ./para.in (or argv[1]) and the image it names,
// prints the parameter block, runs iterate / chkConverge until error <= eps, appends
// Results.dat, prints the Walltime line and writes the field files.
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "piks3d_gpu.h"

int main(int argc, char **argv) {
  const char *para = argc > 1 ? argv[1] : "para.in";
  piks_params p;
  char image[512] = {0};
  if (piks_read_params(para, &p, image, sizeof image)) {
    std::printf(" %s\n", piks_last_error());
    return 1;
  }
  std::printf(" ========== Parameters ================\n");
  std::printf(" imageFileName = %s\n", image);
  std::printf(" Nx = %d\n Ny = %d\n Nz = %d\n", p.Nx + 2 * p.fluidlayer, p.Ny, p.Nz);
  std::printf(" wallExtOrder = %d\n fluidlayer = %d\n Ref_L = %.15g\n", p.wallExtOrder, p.fluidlayer, p.Ref_L);
  std::printf(" Nc_fundamental = %d\n halfRange = %s\n", p.Nc_fundamental, p.halfRange ? "T" : "F");
  std::printf(" maxStep = %d\n chkConvergeStep = %d\n saveStep = %d\n eps = %.15g\n", p.maxStep, p.chkConvergeStep,
              p.saveStep, p.eps);
  std::printf(" saveLast = %s\n saveFormat = %d\n", p.saveLast ? "T" : "F", p.saveFormat);
  std::printf(" Kn = %.15g\n pressDrop = %.15g\n accom = %.15g\n", p.Kn, p.pressDrop, p.accom);
  std::printf(" ======================================\n");
  if (p.mpi_xdim * p.mpi_ydim * p.mpi_zdim != 1)
    std::printf(" note: mpi_xdim*mpi_ydim*mpi_zdim = %d ignored; the GPU solve is one domain\n",
                p.mpi_xdim * p.mpi_ydim * p.mpi_zdim);
  FILE *fh = std::fopen(image, "rb");
  if (!fh) { std::printf(" cannot open image file %s\n", image); return 1; }
  std::vector<uint8_t> raw;
  uint8_t buf[1 << 16];
  size_t n;
  while ((n = std::fread(buf, 1, sizeof buf, fh)) > 0) raw.insert(raw.end(), buf, buf + n);
  std::fclose(fh);
  piks_ctx *ctx = nullptr;
  if (piks_create(&p, 0, &ctx) || piks_setup_physical_grid(ctx, raw.data(), (int64_t)raw.size())) {
    std::printf(" %s\n", piks_last_error());
    return 1;
  }
  int64_t info[10];
  piks_get_info(ctx, info, 10);
  std::printf(" nWall =  %lld\n", (long long)info[5]);
  int32_t steps = 0;
  double perm = 0, secs = 0;
  if (piks_run(ctx, "Results.dat", ".", 1, &steps, &perm, &secs)) {
    std::printf(" %s\n", piks_last_error());
    piks_destroy(ctx);
    return 1;
  }
  piks_destroy(ctx);
  return 0;
}
