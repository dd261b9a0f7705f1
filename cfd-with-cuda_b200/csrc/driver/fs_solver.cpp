// fs_solver: command-line driver with the reference program's contract
// (main and timeLoop of blascoCodinaHuerta.cpp:383-521, 2815-3120):
// reads the problem name from ProblemName.txt (or argv[1]), solves
// <name>.inp, prints the same monitor table and writes <name>.dat (Tecplot)
// at the start, every 1000 steps, at t_final, at steady state and at exit.
// isRestart = 1 in the deck reads <name>_restart.dat.
//
// Solver options (not part of the deck, so the deck stays unchanged):
//   CFD_PRECISION=fp64|mixed  CFD_CG_RTOL=<x>  CFD_CG_WARM=0|1
//   CFD_NGP=8|27  CFD_DEVICE=<n>  CFD_MAXSTEPS=<n>  CFD_DETERMINISTIC=0|1
//   CFD_PRECOND=jacobi|twolevel|learned
//   CFD_UNET=<weight file> (learned; default weights/unet_cavity.bin beside
//     the bin/ folder of this program)
//   CFD_FCG_NET_ITERS=<n> (learned; network in the first n iterations of a
//     pressure solve, 0 = every iteration; default 1)
//   CFD_PGRID=nx,ny,nz (twolevel / learned: the structured grid of the
//     pressure nodes, identity numbering, when they do not form a cube)
#include <unistd.h>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <string>

#include "../../../include/cfdfs.h"

static double now() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// weights/unet_cavity.bin next to the bin/ folder that holds this program
static std::string default_weights() {
  char buf[4096];
  const ssize_t n = readlink("/proc/self/exe", buf, sizeof(buf) - 1);
  if (n <= 0) return "unet_cavity.bin";
  buf[n] = 0;
  std::string exe(buf);
  return exe.substr(0, exe.rfind('/')) + "/../weights/unet_cavity.bin";
}

static int check(cfd_ctx* c, int rc, const char* what) {
  if (rc != CFD_OK) {
    std::fprintf(stderr, "ERROR in %s (%d): %s\n", what, rc, c ? cfd_last_error(c) : "");
    std::exit(1);
  }
  return rc;
}

int main(int argc, char** argv) {
  std::printf("\n\n*********************************************************");
  std::printf("\n*    3D Unsteady Incompressible Navier-Stokes Solver    *");
  std::printf("\n*        Formulation of Blasco, Codina & Huerta         *");
  std::printf("\n*          fractional step, hex27/hex8, B200            *");
  std::printf("\n*********************************************************\n\n");
  std::string name;
  if (argc > 1) {
    name = argv[1];
  } else {
    std::ifstream pn("ProblemName.txt");
    pn >> name;
  }
  if (name.empty()) {
    std::fprintf(stderr, "no problem name (ProblemName.txt or argv[1])\n");
    return 1;
  }
  const char* dev = std::getenv("CFD_DEVICE");
  cfd_ctx* c = nullptr;
  check(nullptr, cfd_create(&c, dev ? std::atoi(dev) : -1), "cfd_create");
  cfd_options o;
  cfd_default_options(&o);
  if (const char* p = std::getenv("CFD_PRECISION")) o.precision = std::strcmp(p, "mixed") == 0 ? CFD_MIXED : CFD_FP64;
  if (const char* p = std::getenv("CFD_CG_RTOL")) o.cg_rtol = std::atof(p);
  if (const char* p = std::getenv("CFD_CG_WARM")) o.cg_warm = std::atoi(p);
  if (const char* p = std::getenv("CFD_NGP")) o.ngp_override = std::atoi(p);
  if (const char* p = std::getenv("CFD_PRECOND"))
    o.precond = std::strcmp(p, "twolevel") == 0  ? CFD_PC_TWOLEVEL
                : std::strcmp(p, "learned") == 0 ? CFD_PC_LEARNED
                                                 : CFD_PC_JACOBI;
  if (o.precond == CFD_PC_LEARNED) o.fcg_net_iters = 1;
  if (const char* p = std::getenv("CFD_FCG_NET_ITERS")) o.fcg_net_iters = std::atoi(p);
  int pgrid[3] = {0, 0, 0};
  bool have_pgrid = false;
  if (const char* p = std::getenv("CFD_PGRID"))
    have_pgrid = std::sscanf(p, "%d,%d,%d", &pgrid[0], &pgrid[1], &pgrid[2]) == 3;
  if (const char* p = std::getenv("CFD_DETERMINISTIC")) o.deterministic = std::atoi(p) != 0;
  long maxsteps = -1;
  if (const char* p = std::getenv("CFD_MAXSTEPS")) maxsteps = std::atol(p);
  check(c, cfd_set_options(c, &o), "cfd_set_options");

  double t0 = now(), t;
  t = now();
  check(c, cfd_load_inp(c, (name + ".inp").c_str()), "cfd_load_inp");
  std::printf("readInputFile() + mesh preprocessing + upload took %8.3f seconds.\n", now() - t);
  cfd_problem_info info;
  cfd_info(c, &info);
  std::ifstream rs((name + "_restart.dat").c_str());
  bool restart = false;
  {
    std::ifstream in((name + ".inp").c_str());
    std::string line;
    while (std::getline(in, line))
      if (line.rfind("isRestart", 0) == 0) {
        restart = std::atoi(line.substr(line.find(':') + 1).c_str()) == 1;
        break;
      }
  }
  if (restart) check(c, cfd_read_restart(c, (name + "_restart.dat").c_str()), "cfd_read_restart");
  check(c, cfd_write_tecplot(c, (name + ".dat").c_str(), name.c_str()), "cfd_write_tecplot");
  t = now();
  check(c, cfd_step0(c), "cfd_step0");
  if (have_pgrid) check(c, cfd_set_pressure_grid(c, pgrid, nullptr), "cfd_set_pressure_grid");
  if (o.precond == CFD_PC_LEARNED) {
    const char* w = std::getenv("CFD_UNET");
    const std::string wpath = w ? std::string(w) : default_weights();
    check(c, cfd_unet_load(c, wpath.c_str(), have_pgrid ? pgrid : nullptr), "cfd_unet_load");
  }
  std::printf("step0()                took  %8.3f seconds.\n", now() - t);
  std::printf("\n NN = %d\n NNp = %d\n sparseM_NNZ = %lld\n sparseG_NNZ = %lld\n NNZ of Z = %lld\n", info.NN,
              info.NNp, 3 * info.nnzK, 3 * info.nnzG, info.nnzZ);
  std::printf("\n\nMonitoring node is %d\n\n\n", info.monPoint);
  std::printf("Time step  Iter     Time       u_monitor     v_monitor     w_monitor     p_monitor     TimeSpend      maxAcc \n");
  std::printf("-------------------------------------------------------------------------------------------------------------\n");
  long steps = 0;
  while (true) {
    cfd_info(c, &info);
    if (!(info.timeT < info.t_final)) break;
    if (maxsteps >= 0 && steps >= maxsteps) break;
    double ts = now();
    check(c, cfd_begin_step(c), "cfd_begin_step");
    int iter;
    for (iter = 1; iter <= info.maxIter; iter++) {
      check(c, cfd_convect(c), "cfd_convect");
      check(c, cfd_step1(c, iter), "cfd_step1");
      check(c, cfd_step2(c, iter, nullptr), "cfd_step2");
      check(c, cfd_step3(c, iter), "cfd_step3");
      int conv = 0;
      check(c, cfd_check_iter(c, info.tolerance, &conv, nullptr), "cfd_check_iter");
      if (conv) break;
      cfd_rotate(c);
      check(c, cfd_k_times_acc(c), "cfd_k_times_acc");
    }
    double maxAcc = 0;
    int steady = 0;
    check(c, cfd_check_steady(c, info.convergence, &maxAcc, &steady), "cfd_check_steady");
    check(c, cfd_end_step(c), "cfd_end_step");
    steps++;
    double mon[4];
    check(c, cfd_get_monitor(c, -1, mon), "cfd_get_monitor");
    cfd_info(c, &info);
    std::printf("%6d  %6d  %10.5f  %12.5f  %12.5f  %12.5f  %12.5f %12.5f %12.5f\n", info.timeN, iter, info.timeT,
                mon[0], mon[1], mon[2], mon[3], now() - ts, maxAcc);
    if (steady) {
      check(c, cfd_write_tecplot(c, (name + ".dat").c_str(), name.c_str()), "cfd_write_tecplot");
      break;
    }
    if (info.timeN % 1000 == 0 || std::fabs(info.timeT - info.t_final) < 1e-10)
      check(c, cfd_write_tecplot(c, (name + ".dat").c_str(), name.c_str()), "cfd_write_tecplot");
  }
  std::printf("\nTotal run took %10.3f seconds.\n", now() - t0);
  std::printf("\nThe program is terminated successfully.\n\n\n");
  check(c, cfd_write_tecplot(c, (name + ".dat").c_str(), name.c_str()), "cfd_write_tecplot");
  cfd_destroy(c);
  return 0;
}
