// Field writers of the drop-in: the files PIKS3D's output module writes for one process
// (output.F90:166-360): Field_000.vti + Field.pvti (saveFormat 1), Field_000.dat
// (Tecplot, 2) and Field_000.vtk (legacy VTK, 3). Values are Rho+1 and U at fluid voxels,
// zeros elsewhere, in ES15.6. List-directed header lines follow gfortran's layout.
#include <cstdio>
#include <string>

#include "piks_internal.h"

namespace piks {

void write_fields(const Setup &s, const Geometry &g, const double *rho, const double *ux,
                  const double *uy, const double *uz, const char *dir, int format,
                  std::string &err, bool &ok) {
  ok = true;
  const std::string d = dir;
  const int Nx = g.Nx, Ny = g.Ny, Nz = g.Nz;
  auto at = [&](int i, int j, int k) { return (size_t)(i - 1) + (size_t)(j - 1) * Nx + (size_t)(k - 1) * Nx * Ny; };
  auto fluid = [&](int i, int j, int k) { return g.label[g.ghost_index(i, j, k)] == L_FLUID; };
  auto open = [&](const std::string &name) -> FILE * {
    FILE *fh = std::fopen((d + "/" + name).c_str(), "w");
    if (!fh) { ok = false; err = "Error: Unable to open output file " + d + "/" + name; }
    return fh;
  };
  if (format == 1) {
    FILE *fh = open("Field_000.vti");
    if (!fh) return;
    std::fprintf(fh, "<?xml version=\"1.0\"?>\n<VTKFile type=\"ImageData\">\n");
    std::fprintf(fh, "<ImageData WholeExtent=\"%4d%4d%4d%4d%4d%4d \" Origin=\"0 0 0\" Spacing=\"1 1 1\">\n", 0, Nx, 0, Ny, 0, Nz);
    std::fprintf(fh, "<Piece Extent=\"%4d%4d%4d%4d%4d%4d\">\n", 0, Nx, 0, Ny, 0, Nz);
    std::fprintf(fh, "<CellData Scalars=\"flag Rho\" Vectors =\"U\">\n");
    std::fprintf(fh, "<DataArray type=\"Int32\" Name=\"flag\" format=\"ascii\">\n");
    for (int k = 1; k <= Nz; ++k)
      for (int j = 1; j <= Ny; ++j)
        for (int i = 1; i <= Nx; ++i) std::fprintf(fh, "%2d\n", (int)g.label[g.ghost_index(i, j, k)]);
    std::fprintf(fh, "</DataArray>\n<DataArray type=\"Float32\" Name=\"Rho\" format=\"ascii\">\n");
    for (int k = 1; k <= Nz; ++k)
      for (int j = 1; j <= Ny; ++j)
        for (int i = 1; i <= Nx; ++i)
          std::fprintf(fh, "%s\n", fortran_es15_6(fluid(i, j, k) ? rho[at(i, j, k)] + 1.0 : 0.0).c_str());
    std::fprintf(fh, "</DataArray>\n<DataArray type=\"Float32\" Name=\"U\" format=\"ascii\" NumberOfComponents=\"3\">\n");
    for (int k = 1; k <= Nz; ++k)
      for (int j = 1; j <= Ny; ++j)
        for (int i = 1; i <= Nx; ++i) {
          bool f = fluid(i, j, k);
          size_t q = at(i, j, k);
          std::fprintf(fh, "%s%s%s\n", fortran_es15_6(f ? ux[q] : 0.0).c_str(), fortran_es15_6(f ? uy[q] : 0.0).c_str(),
                       fortran_es15_6(f ? uz[q] : 0.0).c_str());
        }
    std::fprintf(fh, "</DataArray>\n</CellData>\n</Piece>\n</ImageData>\n</VTKFile>\n");
    std::fclose(fh);
    fh = open("Field.pvti");
    if (!fh) return;
    std::fprintf(fh, "<?xml version=\"1.0\"?>\n<VTKFile type=\"PImageData\">\n");
    std::fprintf(fh, "<PImageData WholeExtent=\"%4d%4d%4d%4d%4d%4d \" Origin=\"0 0 0\" Spacing=\"1 1 1\">\n", 0, Nx, 0, Ny, 0, Nz);
    std::fprintf(fh, "<PCellData Scalars=\"flag Rho\" Vectors =\"U\">\n");
    std::fprintf(fh, "<DataArray type=\"Int32\" Name=\"flag\" format=\"ascii\"/>\n");
    std::fprintf(fh, "<DataArray type=\"Float32\" Name=\"Rho\" format=\"ascii\"/>\n");
    std::fprintf(fh, "<DataArray type=\"Float32\" Name=\"U\" format=\"ascii\" NumberOfComponents=\"3\"/>\n");
    std::fprintf(fh, "</PCellData>\n");
    std::fprintf(fh, "<Piece Extent=\"%4d%4d%4d%4d%4d%4d\" Source=\"Field_000.vti\"/>\n", 0, Nx, 0, Ny, 0, Nz);
    std::fprintf(fh, "</PImageData>\n</VTKFile>\n");
    std::fclose(fh);
  } else if (format == 2) {
    FILE *fh = open("Field_000.dat");
    if (!fh) return;
    std::fprintf(fh, "  TITLE=\" Field\"\n  VARIABLES=x,y,z,flag,Rho,Ux,Uy,Uz\n");
    std::fprintf(fh, " ZONE T=\"proc000\", I=%8d, J=%8d, K=%8d F=POINT\n", Nx, Ny, Nz);
    for (int k = 1; k <= Nz; ++k)
      for (int j = 1; j <= Ny; ++j)
        for (int i = 1; i <= Nx; ++i) {
          bool f = fluid(i, j, k);
          size_t q = at(i, j, k);
          std::fprintf(fh, "%10d%10d%10d%10d%s%s%s%s\n", i, j, k, f ? 0 : 1, fortran_es15_6(f ? rho[q] + 1.0 : 0.0).c_str(),
                       fortran_es15_6(f ? ux[q] : 0.0).c_str(), fortran_es15_6(f ? uy[q] : 0.0).c_str(),
                       fortran_es15_6(f ? uz[q] : 0.0).c_str());
        }
    std::fclose(fh);
  } else if (format == 3) {
    FILE *fh = open("Field_000.vtk");
    if (!fh) return;
    std::fprintf(fh, "# vtk DataFile Version 2.0\nDVM MPI\nASCII\n\nDATASET STRUCTURED_POINTS\n");
    std::fprintf(fh, " DIMENSIONS%12d%12d%12d\n", Nx, Ny, Nz);
    std::fprintf(fh, " ORIGIN%12d%12d%12d\n", 1, 1, 1);
    std::fprintf(fh, " SPACING%12d%12d%12d\n\n", 1, 1, 1);
    std::fprintf(fh, " POINT_DATA%12d\n\n", Nx * Ny * Nz);
    std::fprintf(fh, "SCALARS Rho double\nLOOKUP_TABLE default\n");
    for (int k = 1; k <= Nz; ++k)
      for (int j = 1; j <= Ny; ++j)
        for (int i = 1; i <= Nx; ++i)
          std::fprintf(fh, "%s\n", fortran_es15_6(fluid(i, j, k) ? rho[at(i, j, k)] + 1.0 : 0.0).c_str());
    std::fprintf(fh, "\nVECTORS Velocity double\n");
    for (int k = 1; k <= Nz; ++k)
      for (int j = 1; j <= Ny; ++j)
        for (int i = 1; i <= Nx; ++i) {
          bool f = fluid(i, j, k);
          size_t q = at(i, j, k);
          std::fprintf(fh, "%s%s%s\n", fortran_es15_6(f ? ux[q] : 0.0).c_str(), fortran_es15_6(f ? uy[q] : 0.0).c_str(),
                       fortran_es15_6(f ? uz[q] : 0.0).c_str());
        }
    std::fclose(fh);
  } else {
    ok = false;
    err = "saveFormat must be 1, 2 or 3";
  }
  (void)s;
}

}  // namespace piks
