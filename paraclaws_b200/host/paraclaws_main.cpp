// paraclaws_main.cpp -- the host program of the reference (main.f90) above the C ABI.
//
// Reads control.in and custom.in from the working directory (utility/MOD_IO.f90:25-109),
// sets the initial condition (the dam-break example's set_initial_conditions, or
// initial_state.bin for custom.in initial_condition = 0), and runs the main loop of
// main.f90:193-283 one C-ABI call per reference routine, printing the reference's console lines
// (main.f90:60-61).  With --device-loop the whole loop runs on the device (pcl_advance).
//
// Output: output/final_state.bin (the padded state in the reference layout, raw float64) and
// output/steps.csv (dt used, CFL, time, next dt, ierr, snapshot index per attempted step).
// With --snapshots also writeData's files at t0 and at every snapshot time
// (output/<time>/rank_0/qout.dat and aout.dat, utility/MOD_IO.f90:397-460); in the device loop
// the run pauses at each snapshot time (pcl_advance_to_snapshot) and the files are formatted
// while the next stretch runs.
#include <sys/stat.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "paraclaws_b200.h"

static int fail(const char* where, int rc) {
  std::fprintf(stderr, "paraclaws: %s: %s (%d)\n", where, pcl_status_string(rc), rc);
  return 1;
}

// examples/2D_dam_break/cartesian/SMOD_set_initial_conditions.f90:34-46 on the padded block,
// with the cell centres of domain/SMOD_mesh_manipulation.f90:50-51 (identity mapping)
static void dam_break_ic(const pcl_solver_control& c, std::vector<double>& q) {
  const int ni = c.m_xi + 4, nj = c.m_eta + 4;
  const double dxi = (c.xi_max - c.xi_min) / c.m_xi, deta = (c.eta_max - c.eta_min) / c.m_eta;
  q.assign((size_t)3 * ni * nj, 0.0);
  for (int j = -1; j <= c.m_eta + 2; ++j)
    for (int i = -1; i <= c.m_xi + 2; ++i) {
      double x = c.xi_min + (double)(i - 1) * dxi + dxi / 2;
      double y = c.eta_min + (double)(j - 1) * deta + deta / 2;
      if (c.dam_x0 != 0.0) x = x - c.dam_x0;
      if (c.dam_y0 != 0.0) y = y - c.dam_y0;
      const size_t k = ((size_t)(j + 1) * ni + (i + 1)) * 3;
      q[k] = std::sqrt(x * x + y * y) < c.dam_radius ? c.dam_h_in : c.dam_h_out;
    }
}

int main(int argc, char** argv) {
  bool device_loop = false, snapshots = false;
  int device = 0;
  for (int a = 1; a < argc; ++a) {
    if (!std::strcmp(argv[a], "--device-loop")) device_loop = true;
    else if (!std::strcmp(argv[a], "--snapshots")) snapshots = true;
    else if (!std::strcmp(argv[a], "--device") && a + 1 < argc) device = std::atoi(argv[++a]);
  }
  pcl_solver_control c;
  int rc = pcl_read_solver_control("control.in", "custom.in", &c);
  if (rc) return fail("read_solver_control", rc);
  pcl_ctx* ctx = nullptr;
  if ((rc = pcl_create(&c, device, &ctx))) return fail("pcl_create", rc);
  std::vector<double> q;
  if (c.initial_condition == 0) {
    q.resize((size_t)pcl_state_doubles(ctx));
    FILE* f = std::fopen("initial_state.bin", "rb");
    if (!f || std::fread(q.data(), sizeof(double), q.size(), f) != q.size()) {
      std::fprintf(stderr, "paraclaws: cannot read initial_state.bin\n");
      return 1;
    }
    std::fclose(f);
  } else {
    dam_break_ic(c, q);
  }
  if ((rc = pcl_upload_state(ctx, q.data()))) return fail("upload_state", rc);
  if ((rc = pcl_update_rank_boundaries(ctx))) return fail("update_rank_boundaries", rc);
  mkdir("output", 0755);
  FILE* log = std::fopen("output/steps.csv", "w");
  std::fprintf(log, "dt,cfl,time,dt_next,ierr,snapshot\n");
  double time = 0, dt = 0, dtp = 0, cfl = 0;
  pcl_get_time(ctx, &time);
  std::printf("paraCLAWs - time: %10.8f current dt: %10.8f CFL(max)=%10.5f next dt: %10.8f => snapshot: %4d\n",
              time, c.dt_initial, 0.0, c.dt_initial, 0);
  long long accepted = 0;
  if (snapshots && (rc = pcl_write_snapshot(ctx, "output", 0))) return fail("write_snapshot", rc);  // main.f90:178
  if (device_loop) {
    pcl_run_stats st;
    if (snapshots) {
      for (;;) {
        if ((rc = pcl_advance_to_snapshot(ctx, &st))) return fail("advance_to_snapshot", rc);
        const bool end = st.done || st.time >= c.t_final;
        if (st.time >= c.t_final || !end) {
          std::printf("paraCLAWs - time: %10.8f current dt: %10.8f CFL(max)=%10.5f next dt: %10.8f => snapshot: %4d\n",
                      st.time, st.dt_previous, st.cfl, st.dt, st.snapshot_index - 1);
          if ((rc = pcl_write_snapshot(ctx, "output", 0))) return fail("write_snapshot", rc);
        }
        if (end) break;
      }
    } else if ((rc = pcl_advance(ctx, 0, &st))) {
      return fail("advance", rc);
    }
    long long n = 0;
    pcl_get_step_log(ctx, nullptr, 0, &n);
    std::vector<pcl_step_record> recs((size_t)n);
    pcl_get_step_log(ctx, recs.data(), n, &n);
    for (const auto& r : recs)
      std::fprintf(log, "%.17g,%.17g,%.17g,%.17g,%d,%d\n", r.dt, r.cfl, r.time, r.dt_next, r.ierr, r.snapshot_index);
    accepted = st.accepted;
    time = st.time;
  } else {
    const int nsnap = c.number_of_snapshots < 1 ? 1 : c.number_of_snapshots;
    while (time < c.t_final) {                                     // main.f90:193
      if (c.max_accepted_steps > 0 && accepted >= c.max_accepted_steps) break;
      double dt_used = 0;
      pcl_get_dt(ctx, &dt_used);
      int ierr = 0;
      if ((rc = pcl_solve_dimensional_split(ctx, &ierr))) return fail("solve_dimensional_split", rc);  // :210
      pcl_get_cfl(ctx, &cfl);
      int snap = 0;
      if (ierr < 0) {                                              // :213-233
        std::printf("WARNING: time step rejected!\n");
        if ((rc = pcl_update_time(ctx, 0))) return fail("update_time", rc);
        pcl_restore_solution(ctx);
        pcl_reset_cfl(ctx);
        pcl_get_snapshot_index(ctx, &snap);
        pcl_get_time(ctx, &time);
        pcl_get_dt(ctx, &dt);
      } else {
        pcl_integrate_source_term(ctx);                            // :238
        pcl_update_rank_boundaries(ctx);                           // :246
        if ((rc = pcl_update_time(ctx, 1))) return fail("update_time", rc);  // :251
        pcl_get_time(ctx, &time);
        pcl_get_dt(ctx, &dt);
        pcl_get_previous_dt(ctx, &dtp);
        pcl_get_snapshot_index(ctx, &snap);
        double ts = 0;
        pcl_get_snapshot_time(ctx, snap <= nsnap ? snap : nsnap, &ts);
        if (snap <= nsnap && time >= ts) {                         // :256-268
          std::printf("paraCLAWs - time: %10.8f current dt: %10.8f CFL(max)=%10.5f next dt: %10.8f => snapshot: %4d\n",
                      time, dtp, cfl, dt, snap);
          if (snapshots && (rc = pcl_write_snapshot(ctx, "output", 0))) return fail("write_snapshot", rc);  // :260
          pcl_advance_snapshot_index(ctx);
          snap += 1;
        } else {
          std::printf("paraCLAWs - time: %10.8f current dt: %10.8f CFL(max)=%10.5f next dt: %10.8f\n", time, dtp,
                      cfl, dt);
        }
        pcl_reset_cfl(ctx);                                        // :275
        accepted += 1;
      }
      std::fprintf(log, "%.17g,%.17g,%.17g,%.17g,%d,%d\n", dt_used, cfl, time, dt, ierr, snap);
    }
  }
  std::fclose(log);
  if (snapshots && (rc = pcl_snapshot_wait(ctx))) return fail("snapshot_wait", rc);
  if ((rc = pcl_download_state(ctx, q.data()))) return fail("download_state", rc);
  FILE* f = std::fopen("output/final_state.bin", "wb");
  std::fwrite(q.data(), sizeof(double), q.size(), f);
  std::fclose(f);
  pcl_destroy(ctx);
  std::printf("PROGRAM FINISHED SUCCESSFULLY: %lld accepted steps, time %.17g\n", accepted, time);
  return 0;
}
