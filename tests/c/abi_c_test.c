/* The C ABI from plain C (C99, no GPU): the entry points that need no
 * device -- version and status strings, the built-in integrand programs,
 * checkpoint write / info / read and its integrity check, the VTK writer.
 * Usage: abi_c_test <scratch directory>.  Prints PASS lines; exit 0 when all pass. */
#include <stdio.h>
#include <string.h>

#include "gridcalc_b200.h"

static int failures = 0;

static void check(int ok, const char* what) {
  printf("%s %s\n", ok ? "PASS" : "FAIL", what);
  if (!ok) failures++;
}

int main(int argc, char** argv) {
  char path[4096], vtk[4096], meta[64];
  double field[3 * 4 * 5], back[3 * 4 * 5];
  gc_grid g = {5, 4, 3, 0.5, 0.25, 2.0}, g2;
  gc_dtype dt;
  int32_t comps;
  size_t meta_len, i;
  gc_integrand fe = {GC_INTEGRAND_CH_FREE_ENERGY, 0.8};
  gc_program prog;
  FILE* f;
  unsigned char byte;

  if (argc < 2) return 2;
  snprintf(path, sizeof path, "%s/state.gcb", argv[1]);
  snprintf(vtk, sizeof vtk, "%s/psi.vtk", argv[1]);

  check(gc_version() != NULL && gc_version()[0] != '\0', "gc_version");
  check(strcmp(gc_status_string(GC_ERR_IO), "GC_ERR_IO") == 0 &&
            strcmp(gc_status_string(GC_ERR_AXIS_EXTENT), "GC_ERR_AXIS_EXTENT") == 0,
        "gc_status_string");

  check(gc_integrand_program(&fe, &prog) == GC_OK && prog.components == 1 && prog.arity == 2 &&
            prog.n_instr == 21 && prog.instr[prog.n_instr - 3].op == GC_OPC_CONST &&
            prog.instr[prog.n_instr - 3].value == 0.5 * 0.8,
        "gc_integrand_program (free energy, kappa 0.5 * 0.8 as a constant)");

  for (i = 0; i < sizeof field / sizeof field[0]; ++i) field[i] = 0.1 * (double)i - 2.0;
  check(gc_write_checkpoint(&g, GC_F64, 1, field, path, "{\"step\": 12}") == GC_OK, "gc_write_checkpoint");
  check(gc_checkpoint_info(path, &g2, &dt, &comps, &meta_len) == GC_OK && g2.nx == 5 && g2.ny == 4 && g2.nz == 3 &&
            g2.hx == 0.5 && g2.hy == 0.25 && g2.hz == 2.0 && dt == GC_F64 && comps == 1 && meta_len == 12,
        "gc_checkpoint_info");
  memset(back, 0, sizeof back);
  check(gc_read_checkpoint(path, back, sizeof back, meta, sizeof meta) == GC_OK &&
            memcmp(back, field, sizeof field) == 0 && strcmp(meta, "{\"step\": 12}") == 0,
        "gc_read_checkpoint round trip");

  /* One flipped bit of the stored spacing hx fails the load. */
  f = fopen(path, "r+b");
  if (f && fseek(f, 32, SEEK_SET) == 0 && fread(&byte, 1, 1, f) == 1 && fseek(f, 32, SEEK_SET) == 0) {
    byte ^= 0x10;
    fwrite(&byte, 1, 1, f);
  }
  if (f) fclose(f);
  check(gc_read_checkpoint(path, back, sizeof back, meta, sizeof meta) == GC_ERR_IO &&
            strstr(gc_last_error(), "checksum") != NULL,
        "corrupted header detected");

  check(gc_write_vtk(&g, GC_F64, field, vtk, "psi", GC_VTK_ASCII) == GC_OK, "gc_write_vtk");
  g.nx = 0;
  check(gc_write_vtk(&g, GC_F64, field, vtk, "psi", GC_VTK_ASCII) == GC_ERR_INVALID_ARG &&
            strstr(gc_last_error(), "extents") != NULL,
        "invalid grid rejected with the reference's message");
  return failures ? 1 : 0;
}
