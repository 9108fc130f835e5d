// Binding check: TEST INFRASTRUCTURE ONLY.
//
// Compiles the drop-in binding include/sbd_tpb_sbd.hpp the way a maintainer of the reference would
// (against the reference's own headers, here with the single-rank MPI shim) and runs the app's flow
// (apps/chemistry_tpb_selected_basis_diagonalization/main.cc:124-191: LoadFCIDump, LoadAlphaDets +
// sort_bitarray, bdet = adet) through both sbd::tpb::diag (tpb/sbdiag.h:139-151, the reference on the
// host) and sbd_b200::diag (the library on the GPU) with the same settings.  Prints one line of
// key=value pairs: the two energies, the largest differences of density, 1-RDM and 2-RDM entries,
// and whether the carry-over strings are equal (as sets, and in the same order).
// Usage: binding_check --fcidump F --adetfile A [--iteration I] [--block B] [--tolerance T]
//                      [--rdm] [--carryover_type K --carryover_threshold X] [--init I --seed S]
//                      [--loadname NAME] [--savename NAME] [--skip_reference]
#include <chrono>
#include <cmath>
#include <cstdio>
#include <algorithm>
#include <deque>
#include <iostream>
#include <string>
#include <unistd.h>
#include <vector>

#include "mpi.h"
#include "sbd/sbd.h"
#include "sbd_tpb_sbd.hpp"

namespace {

double max_diff(const std::vector<double> &x, const std::vector<double> &y) {
  if (x.size() != y.size()) return INFINITY;
  double m = 0.0;
  for (size_t i = 0; i < x.size(); ++i) m = std::max(m, std::fabs(x[i] - y[i]));
  return m;
}

double max_diff(const std::vector<std::vector<double>> &x, const std::vector<std::vector<double>> &y) {
  if (x.size() != y.size()) return INFINITY;
  double m = 0.0;
  for (size_t k = 0; k < x.size(); ++k) m = std::max(m, max_diff(x[k], y[k]));
  return m;
}

}  // namespace

int main(int argc, char **argv) {
  std::string fcidumpfile, adetfile, loadname, savename;
  bool skip_reference = false;
  sbd::tpb::SBD s;
  for (int i = 1; i < argc; ++i) {
    std::string a(argv[i]);
    if (a == "--fcidump") fcidumpfile = argv[++i];
    else if (a == "--adetfile") adetfile = argv[++i];
    else if (a == "--iteration") s.max_it = std::atoi(argv[++i]);
    else if (a == "--block") s.max_nb = std::atoi(argv[++i]);
    else if (a == "--tolerance") s.eps = std::atof(argv[++i]);
    else if (a == "--rdm") s.do_rdm = 1;
    else if (a == "--init") s.init = std::atoi(argv[++i]);
    else if (a == "--seed") s.seed = std::strtoull(argv[++i], nullptr, 10);
    else if (a == "--carryover_type") s.carryover_type = std::atoi(argv[++i]);
    else if (a == "--carryover_threshold") s.threshold = std::atof(argv[++i]);
    else if (a == "--loadname") loadname = argv[++i];
    else if (a == "--savename") savename = argv[++i];
    else if (a == "--skip_reference") skip_reference = true;
    else {
      std::fprintf(stderr, "binding_check: unknown argument %s\n", a.c_str());
      return 2;
    }
  }
  int provided;
  MPI_Init_thread(&argc, &argv, MPI_THREAD_FUNNELED, &provided);
  MPI_Comm comm = MPI_COMM_WORLD;
  sbd::FCIDump fcidump = sbd::LoadFCIDump(fcidumpfile);
  int L = 0;
  for (const auto &[key, value] : fcidump.header)
    if (key == std::string("NORB")) L = std::atoi(value.c_str());
  std::vector<std::vector<size_t>> adet, bdet;
  sbd::LoadAlphaDets(adetfile, adet, s.bit_length, L);
  sbd::sort_bitarray(adet);
  bdet = adet;

  double e_ref = 0.0, e_b200 = 0.0;
  std::vector<double> d_ref, d_b200;
  std::vector<std::vector<size_t>> ca_ref, cb_ref, ca_b200, cb_b200;
  std::vector<std::vector<double>> one_ref, two_ref, one_b200, two_b200;
  double t_ref = 0.0;
  if (!skip_reference) {
    const auto t0 = std::chrono::steady_clock::now();
    sbd::tpb::diag(comm, s, fcidump, adet, bdet, loadname, "", e_ref, d_ref, ca_ref, cb_ref, one_ref, two_ref);
    t_ref = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
  const auto t1 = std::chrono::steady_clock::now();
  try {
    sbd_b200::diag(comm, s, fcidump, adet, bdet, loadname, savename, e_b200, d_b200, ca_b200, cb_b200,
                   one_b200, two_b200);
  } catch (const std::exception &e) {
    std::fprintf(stderr, "sbd_b200::diag: %s\n", e.what());
    MPI_Finalize();
    return 3;
  }
  const double t_b200 = std::chrono::duration<double>(std::chrono::steady_clock::now() - t1).count();
  // carry-over strings: in the same order, and as sets (strings of equal weight, e.g. related by
  // the molecule's spatial symmetry, may be ordered differently by rounding-level differences of
  // the two vectors; the next load of the strings sorts them)
  auto sorted = [](std::vector<std::vector<size_t>> v) {
    std::sort(v.begin(), v.end());
    return v;
  };
  const int co_seq = (int)(ca_ref == ca_b200 && cb_ref == cb_b200);
  const int co_set = (int)(sorted(ca_ref) == sorted(ca_b200) && sorted(cb_ref) == sorted(cb_b200));
  std::printf("e_ref=%.15f e_b200=%.15f density_diff=%.3e rdm1_diff=%.3e rdm2_diff=%.3e "
              "co_equal=%d co_same_order=%d co_a=%zu co_b=%zu co_a_ref=%zu co_b_ref=%zu t_ref=%.3f t_b200=%.3f\n",
              e_ref, e_b200, skip_reference ? 0.0 : max_diff(d_ref, d_b200),
              s.do_rdm && !skip_reference ? max_diff(one_ref, one_b200) : 0.0,
              s.do_rdm && !skip_reference ? max_diff(two_ref, two_b200) : 0.0, co_set, co_seq,
              ca_b200.size(), cb_b200.size(), ca_ref.size(), cb_ref.size(), t_ref, t_b200);
  MPI_Finalize();
  return 0;
}
