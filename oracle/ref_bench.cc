// Reference CPU timing driver: TEST/BENCH INFRASTRUCTURE ONLY.
//
// Times the reference's own CPU sigma (sbd::mult, tpb/mult.h:625-881, OpenMP, one MPI rank via
// the single-rank shim) on a bounded sample of a workload: the first --amax alpha strings (after
// LoadAlphaDets' sort) times all beta strings.  Prints one line of key=value pairs:
//   ndet, helper_s (MakeHelpers + RemakeHelpers, tpb/helper.h:710-1226), hii_s
//   (makeQChamDiagTerms), sigma_s (seconds of each of --reps mult calls), threads.
// Usage: ref_bench --fcidump F --adetfile A [--bdetfile B] [--amax M] [--reps K]
//        ref_bench --parse FILE --norb L [--reps K]
//   times LoadAlphaDets (basic/makedeterminants.h:160-186: read, from_string or DecodeAlphaDets,
//   sort_bitarray) on a string file alone and prints nstrings and parse_s (seconds per call).
#include <chrono>
#include <cmath>
#include <deque>
#include <unistd.h>
#include <cstdio>
#include <iostream>
#include <random>
#include <string>
#include <vector>

#include "mpi.h"
#include "sbd/sbd.h"

int main(int argc, char **argv) {
  std::string fcidumpfile, adetfile, bdetfile;
  size_t amax = 0, bit_length = 20;
  int reps = 1;
  std::string parsefile;
  size_t parse_norb = 0;
  for (int i = 1; i < argc; ++i) {
    std::string a(argv[i]);
    if (a == "--parse") parsefile = argv[++i];
    else if (a == "--norb") parse_norb = std::strtoul(argv[++i], nullptr, 10);
    if (a == "--fcidump") fcidumpfile = argv[++i];
    else if (a == "--adetfile") adetfile = argv[++i];
    else if (a == "--bdetfile") bdetfile = argv[++i];
    else if (a == "--amax") amax = std::strtoul(argv[++i], nullptr, 10);
    else if (a == "--reps") reps = std::atoi(argv[++i]);
  }
  int provided;
  MPI_Init_thread(&argc, &argv, MPI_THREAD_FUNNELED, &provided);
  if (!parsefile.empty()) {
    std::vector<std::vector<size_t>> d;
    std::string ts;
    for (int r = 0; r < reps; ++r) {
      d.clear();
      auto p0 = std::chrono::steady_clock::now();
      sbd::LoadAlphaDets(parsefile, d, bit_length, parse_norb);
      auto p1 = std::chrono::steady_clock::now();
      ts += (r ? "," : "") + std::to_string(std::chrono::duration<double>(p1 - p0).count());
    }
    std::printf("nstrings=%zu parse_s=%s\n", d.size(), ts.c_str());
    MPI_Finalize();
    return 0;
  }
  sbd::FCIDump fcidump = sbd::LoadFCIDump(fcidumpfile);
  int L = 0, N = 0;
  double I0 = 0.0;
  sbd::oneInt<double> I1;
  sbd::twoInt<double> I2;
  sbd::SetupIntegrals(fcidump, L, N, I0, I1, I2);
  std::vector<std::vector<size_t>> adet, bdet;
  sbd::LoadAlphaDets(adetfile, adet, bit_length, L);
  sbd::sort_bitarray(adet);
  if (bdetfile.empty()) bdet = adet;
  else {
    sbd::LoadAlphaDets(bdetfile, bdet, bit_length, L);
    sbd::sort_bitarray(bdet);
  }
  if (amax > 0 && amax < adet.size()) adet.resize(amax);
  MPI_Comm comm = MPI_COMM_WORLD, h_comm, b_comm, t_comm, a_comm;
  sbd::TaskCommunicator(comm, 1, 1, 1, 1, h_comm, b_comm, t_comm, a_comm);
  auto t0 = std::chrono::steady_clock::now();
  std::vector<sbd::TaskHelpers> helper;
  sbd::MakeHelpers(adet, bdet, bit_length, L, helper, h_comm, b_comm, t_comm, 1, 1);
  sbd::RemakeHelpers(adet, bdet, bit_length, L, helper, h_comm, b_comm, t_comm, 1, 1);
  auto t1 = std::chrono::steady_clock::now();
  std::vector<double> hii;
  sbd::makeQChamDiagTerms(adet, bdet, bit_length, L, helper, I0, I1, I2, hii, h_comm, b_comm, t_comm);
  auto t2 = std::chrono::steady_clock::now();
  std::vector<double> win(hii.size()), wout(hii.size());
  std::mt19937_64 g(7);
  std::normal_distribution<double> nd(0.0, 1.0);
  for (auto &x : win) x = nd(g);
  std::printf("ndet=%zu helper_s=%.6f hii_s=%.6f threads=%d sigma_s=", hii.size(),
              std::chrono::duration<double>(t1 - t0).count(),
              std::chrono::duration<double>(t2 - t1).count(), omp_get_max_threads());
  for (int r = 0; r < reps; ++r) {
    std::fill(wout.begin(), wout.end(), 0.0);
    auto s0 = std::chrono::steady_clock::now();
    sbd::mult(hii, win, wout, adet, bdet, bit_length, static_cast<size_t>(L), 1, 1, helper, I0, I1,
              I2, h_comm, b_comm, t_comm);
    auto s1 = std::chrono::steady_clock::now();
    std::printf("%s%.6f", r ? "," : "", std::chrono::duration<double>(s1 - s0).count());
  }
  double cs = 0.0;
  for (double x : wout) cs += x;
  std::printf(" checksum=%.17g\n", cs);
  MPI_Finalize();
  return 0;
}
