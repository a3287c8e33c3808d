/*
 * Step-by-step driver for the CloverLeaf 2D application (an OPS user app,
 * built unchanged from its own sources with clover_leaf.cpp's main renamed).
 *
 * The benchmark needs to time individual hydro steps with warm-up steps
 * excluded, so this harness exposes the app's setup and one hydro step as C
 * entry points.  setup mirrors the start of clover_leaf.cpp's main (ops_init,
 * initialise, the ops_decl_const list, start) and a step is the body of its
 * hydro loop (clover_leaf.cpp:180-199): timestep, PdV predict, accelerate,
 * PdV correct, flux_calc, advection, reset_field, direction switch.
 *
 * The same file builds against this backend and against the reference
 * OpenMP backend, so both are driven through identical calls.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>
#if defined(CLOVER_STEP_CUDA)
#include <cuda_runtime_api.h>
#endif

#define OPS_2D
#include "ops_seq_v2.h"
#include "data.h"
#include "definitions.h"
#include "dumpdats.h"

void initialise();
void field_summary();
void timestep();
void PdV(int predict);
void accelerate();
void flux_calc();
void advection(int);
void reset_field();
void start();

extern double g_small, g_big, dtc_safe, dtu_safe, dtv_safe, dtdiv_safe, dt, clover_time;
extern double end_time;
extern int number_of_states, g_circ, g_point, g_rect, step, advect_x, complete, end_step;
extern FILE *g_out;

extern "C" {

/* Reads clover.in from the current directory. */
__attribute__((visibility("default"))) int clover_step_setup(int argc, char **argv) {
  ops_init(argc, argv, 1);
  initialise();
  ops_decl_const("g_small", 1, "double", &g_small);
  ops_decl_const("g_big", 1, "double", &g_big);
  ops_decl_const("dtc_safe", 1, "double", &dtc_safe);
  ops_decl_const("dtu_safe", 1, "double", &dtu_safe);
  ops_decl_const("dtv_safe", 1, "double", &dtv_safe);
  ops_decl_const("dtdiv_safe", 1, "double", &dtdiv_safe);
  ops_decl_const("field", 1, "field_type", &field);
  ops_decl_const("grid", 1, "grid_type", &grid);
  ops_decl_const("number_of_states", 1, "int", &number_of_states);
  ops_decl_const("states", number_of_states, "state_type", states);
  ops_decl_const("g_circ", 1, "int", &g_circ);
  ops_decl_const("g_point", 1, "int", &g_point);
  ops_decl_const("g_rect", 1, "int", &g_rect);
  ops_decl_const("dt", 1, "double", &dt);
  start();
  return 0;
}

/* Runs n hydro steps; returns the simulated time reached. */
__attribute__((visibility("default"))) double clover_step_run(int n) {
  for (int i = 0; i < n; i++) {
    step = step + 1;
    timestep();
    PdV(TRUE);
    accelerate();
    PdV(FALSE);
    flux_calc();
    advection(step);
    reset_field();
    advect_x = (advect_x == TRUE) ? FALSE : TRUE;
    clover_time = clover_time + dt;
  }
  ops_execute();  // the loops queued after the last reduction (lazy execution)
  return clover_time;
}

/* field_summary of the app (writes the summary line to clover.out). */
__attribute__((visibility("default"))) void clover_step_summary(void) {
  complete = TRUE;
  field_summary();
  fflush(g_out);
}

/* Waits until every step issued so far has finished on the device (the
 * reference's CUDA backend returns from a loop before its kernel ends;
 * this backend's ops_timers flushes its queue and waits for the device). */
__attribute__((visibility("default"))) void clover_step_sync(void) {
#if defined(CLOVER_STEP_CUDA)
  cudaDeviceSynchronize();
#else
  double c, e;
  ops_timers(&c, &e);
#endif
}

__attribute__((visibility("default"))) int clover_step_current(void) { return step; }

/* Every dat of the application (build_field.cpp) written to `path` through
 * ops_dat_fetch_data (apps/dumpdats.h): interiors, the same on every backend. */
__attribute__((visibility("default"))) int clover_step_dump(const char *path) {
  ops_dat all[] = {density0, density1, energy0, energy1, pressure, viscosity, soundspeed,
                   volume, xvel0, xvel1, yvel0, yvel1, vol_flux_x, vol_flux_y, mass_flux_x,
                   mass_flux_y, xarea, yarea, work_array1, work_array2, work_array3,
                   work_array4, work_array5, work_array6, work_array7, cellx, celly, vertexx,
                   vertexy, celldx, celldy, vertexdx, vertexdy, xx, yy};
  return dump_dats(path, all, (int)(sizeof(all) / sizeof(all[0])));
}

/* Moves every dat of the application between the device and host buffers
 * through the public data-access calls: dir 0 fetches each dat's interior
 * into bufs[i], dir 1 sets it from bufs[i].  Returns the dat count (with
 * bufs == NULL: the count, and the byte size of each into sizes). */
__attribute__((visibility("default"))) int clover_step_state(int dir, char **bufs,
                                                             long long *sizes) {
  ops_dat all[] = {density0, density1, energy0, energy1, pressure, viscosity, soundspeed,
                   volume, xvel0, xvel1, yvel0, yvel1, vol_flux_x, vol_flux_y, mass_flux_x,
                   mass_flux_y, xarea, yarea, work_array1, work_array2, work_array3,
                   work_array4, work_array5, work_array6, work_array7, cellx, celly, vertexx,
                   vertexy, celldx, celldy, vertexdx, vertexdy, xx, yy};
  const int n = (int)(sizeof(all) / sizeof(all[0]));
  for (int i = 0; i < n; i++) {
    if (!bufs) {
      int disp[2], ext[2];
      ops_dat_get_extents(all[i], 0, disp, ext);
      if (sizes) sizes[i] = (long long)ext[0] * ext[1] * all[i]->elem_size;
      continue;
    }
    if (dir == 0)
      ops_dat_fetch_data(all[i], 0, bufs[i]);
    else
      ops_dat_set_data(all[i], 0, bufs[i]);
  }
  return n;
}

__attribute__((visibility("default"))) void clover_step_finish(void) {
  fflush(g_out);
  ops_exit();
}

}  // extern "C"
