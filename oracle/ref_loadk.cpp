// Runs the reference's load_permeability (main.cpp:918-1032, compiled with
// LOAD_K_FROM_FILE) on <workdir>/noise.dat and writes the K array it fills
// (nx*ny*nz float64, index i + j*nx + k*nx*ny) to <out>.  Test
// infrastructure: the parity reference for the product's permeability-file
// reader.
//
//   capaz_ref_loadk <workdir> <nx> <ny> <nz> <out>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include <vector>

#include "defines.h"

int main(int argc, char** argv) {
  if (argc != 6) {
    fprintf(stderr, "usage: %s <workdir> <nx> <ny> <nz> <out>\n", argv[0]);
    return 2;
  }
  if (chdir(argv[1]) != 0) {
    perror("chdir");
    return 2;
  }
  consts def;
  memset(&def, 0, sizeof def);
  def.Nx = def.locNx = atoi(argv[2]);
  def.Ny = def.locNy = atoi(argv[3]);
  def.Nz = def.locNz = atoi(argv[4]);
  def.size = def.sizex = def.sizey = def.sizez = 1;
  def.upscale_l = 1.;
  def.K[0] = 1e-12;
  const long n = (long)def.Nx * def.Ny * def.Nz;
  std::vector<double> K(n, 0.);
  load_permeability(K.data(), def);
  FILE* f = fopen(argv[5], "wb");
  if (!f || fwrite(K.data(), sizeof(double), n, f) != (size_t)n) return 3;
  fclose(f);
  return 0;
}
