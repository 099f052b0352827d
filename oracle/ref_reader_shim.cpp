// TEST INFRASTRUCTURE ONLY — never linked into the product library.
//
// Host shim around the reference's own input-file reader (LBM-C
// infile_reader.cu:45-226, class InfileReader) so that the engine's
// lbmc_read_input can be compared with it field by field on the same files.
// oracle/build_ref.sh compiles this file against the reference sources (a
// temporary copy with the lattice selected as macros.cu:11-12 does) into
// oracle/_ref/libref_reader_<lattice>.so; nothing of the reference is copied
// into the repository.
//
// The reader prints its report to std::cout; ref_read_input captures it into
// the caller's buffer.  The structs it fills are zeroed first (the reference
// leaves every field it does not read uninitialised, except C_smag).

#include <cstdio>
#include <cstring>
#include <iostream>
#include <sstream>
#include <string>

#define __device__
#define __constant__
#define __noinline__
#define __global__
#define __host__

#include "macros.cu"
#include "data_types.cuh"
#include "infile_reader.cu"

extern "C" {

// Every field InfileReader sets, in plain C types.
struct ref_input {
  double tau, tau_mrt[15], c_smag, tolerance;
  int length[3], h, dt, forcing, macro_bc, micro_bc, collision_type, init_type;
  int max_t, plot, screen, steady_check;
  int out_u[3], out_rho, out_pressure, interactive, screen_node[3];
  char name[STR_LENGTH], domain_fname[STR_LENGTH], output_fname[STR_LENGTH];
};

int ref_reader_dim(void) { return DIM; }
int ref_reader_str_length(void) { return STR_LENGTH; }

// Reads `path` with the reference's InfileReader; returns DIM.  `report`
// (may be NULL) receives what the reader printed, truncated to report_bytes.
int ref_read_input(const char *path, ref_input *out, char *report, size_t report_bytes) {
  ProjectStrings project;
  DomainConstant dc;
  Timing timer;
  OutputController oc;
  memset(&project, 0, sizeof(project));
  memset(&dc, 0, sizeof(dc));
  memset(&timer, 0, sizeof(timer));
  memset(&oc, 0, sizeof(oc));
  std::ostringstream captured;
  std::streambuf *old = std::cout.rdbuf(captured.rdbuf());
  {
    std::string p(path);
    InfileReader reader(&p[0], &project, &dc, &timer, &oc);
    (void)reader;
  }
  std::cout.rdbuf(old);
  memset(out, 0, sizeof(*out));
  out->tau = dc.tau;
  for (int i = 0; i < Q; i++) out->tau_mrt[i] = dc.tau_mrt[i];
  out->c_smag = dc.c_smag;
  out->tolerance = dc.tolerance;
  for (int d = 0; d < DIM; d++) out->length[d] = dc.length[d];
  out->h = dc.h;
  out->dt = dc.dt;
  out->forcing = dc.forcing;
  out->macro_bc = dc.macro_bc;
  out->micro_bc = dc.micro_bc;
  out->collision_type = dc.collision_type;
  out->init_type = dc.init_type;
  out->max_t = timer.max;
  out->plot = timer.plot;
  out->screen = timer.screen;
  out->steady_check = timer.steady_check;
  for (int d = 0; d < DIM; d++) {
    out->out_u[d] = oc.u[d];
    out->screen_node[d] = oc.screen_node[d];
  }
  out->out_rho = oc.rho;
  out->out_pressure = oc.pressure;
  out->interactive = oc.interactive;
  memcpy(out->name, project.name, STR_LENGTH);
  memcpy(out->domain_fname, project.domain_fname, STR_LENGTH);
  memcpy(out->output_fname, project.output_fname, STR_LENGTH);
  if (report && report_bytes) {
    const std::string s = captured.str();
    const size_t k = s.size() < report_bytes - 1 ? s.size() : report_bytes - 1;
    memcpy(report, s.data(), k);
    report[k] = 0;
  }
  return DIM;
}

}  // extern "C"
