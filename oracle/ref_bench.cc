// Reference CPU timing driver: TEST/BENCH INFRASTRUCTURE ONLY.
//
// Times the reference's own CPU sigma (sbd::mult, tpb/mult.h:625-881, OpenMP, one MPI rank via
// the single-rank shim) on the whole problem of a workload: every alpha and beta string, every
// connection.  Two modes:
//
//   full (default)   --reps K calls of mult over the whole determinant space.
//   bra blocks       --blocks K --rows R (or --target_s T: R chosen so one block call takes about
//                    T seconds, from a probe block of na/200 rows in the middle of the list):
//                    first one call whose alpha bra range is empty (what
//                    mult costs for any range: its N-sized ket copy (Mpi2dSlide through the
//                    single-rank shim) and diagonal pass, tpb/mult.h:676-687), then K calls
//                    each over R consecutive alpha bra strings with all beta strings and ALL
//                    kets, the K blocks spread evenly over the sorted alpha list.  A block call
//                    does exactly the work mult does for those bra rows (their alpha, beta and
//                    alpha-beta connections, tpb/mult.h:717-840) plus the fixed part.  The bra
//                    range is narrowed by pointing the 1-rank TaskHelpers' per-bra-string arrays
//                    (tpb/helper.h:14-67) at the block: their entries are untouched, so each
//                    row's connections are the full problem's; sigma rows land at the start of
//                    the output vector (timing only).
//
// --no_hii fills H_ii with zeros instead of calling makeQChamDiagTerms (tpb/qcham.h:290-340):
// mult's diagonal pass does the same multiply-adds whatever the values, and the diagonal of a
// 4e8-determinant problem takes minutes to build on the host.
//
// The input vector is x_i = ((i * 0x9E3779B97F4A7C15 mod 2^64) >> 11) / 2^53 - 1/2 (cheap to fill
// at 4e8 determinants; mult's work does not depend on the values).
//
// Prints one line of key=value pairs: ndet, na, nb, helper_s (MakeHelpers + RemakeHelpers,
// tpb/helper.h:710-1226), hii_s, threads, then sigma_s (seconds of each full call) or fixed_s,
// rows, block_s (seconds of each block call), block_start (first bra row of each block) and
// block_sum (sum of the output vector after each block call).
// Usage: ref_bench --fcidump F --adetfile A [--bdetfile B] [--reps K] [--no_hii]
//        ref_bench --fcidump F --adetfile A --blocks K (--rows R | --target_s T) [--no_hii]
//        ref_bench --parse FILE --norb L [--reps K]
//   the last times LoadAlphaDets (basic/makedeterminants.h:160-186: read, from_string or
//   DecodeAlphaDets, sort_bitarray) on a string file alone and prints nstrings and parse_s.
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

namespace {

double seconds_since(std::chrono::steady_clock::time_point t0) {
  return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// The per-bra-alpha-string arrays of one task, saved so a block view can be put back.
struct AlphaView {
  size_t start, end;
  size_t *s_len, *d_len;
  std::vector<size_t *> s_sm, d_sm;
  std::vector<int *> s_cran, d_cran;
};

AlphaView save_view(const sbd::TaskHelpers &h) {
  return AlphaView{h.braAlphaStart,        h.braAlphaEnd,         h.SinglesFromAlphaLen,
                   h.DoublesFromAlphaLen,  h.SinglesFromAlphaSM,  h.DoublesFromAlphaSM,
                   h.SinglesAlphaCrAnSM,   h.DoublesAlphaCrAnSM};
}

// Point the task at bra alpha rows [lo, hi) of the saved view (indices relative to its start).
void set_view(sbd::TaskHelpers &h, const AlphaView &v, size_t lo, size_t hi) {
  h.braAlphaStart = v.start + lo;
  h.braAlphaEnd = v.start + hi;
  h.SinglesFromAlphaLen = v.s_len + lo;
  h.DoublesFromAlphaLen = v.d_len + lo;
  auto sub = [&](const auto &src, auto &dst) {
    dst.assign(src.begin() + std::min(lo, src.size()), src.begin() + std::min(hi, src.size()));
  };
  sub(v.s_sm, h.SinglesFromAlphaSM);
  sub(v.d_sm, h.DoublesFromAlphaSM);
  sub(v.s_cran, h.SinglesAlphaCrAnSM);
  sub(v.d_cran, h.DoublesAlphaCrAnSM);
}

void restore_view(sbd::TaskHelpers &h, const AlphaView &v) {
  h.braAlphaStart = v.start;
  h.braAlphaEnd = v.end;
  h.SinglesFromAlphaLen = v.s_len;
  h.DoublesFromAlphaLen = v.d_len;
  h.SinglesFromAlphaSM = v.s_sm;
  h.DoublesFromAlphaSM = v.d_sm;
  h.SinglesAlphaCrAnSM = v.s_cran;
  h.DoublesAlphaCrAnSM = v.d_cran;
}

}  // namespace

int main(int argc, char **argv) {
  std::string fcidumpfile, adetfile, bdetfile;
  size_t bit_length = 20, rows = 0;
  int reps = 1, blocks = 0;
  bool no_hii = false;
  double target_s = 0.0;
  std::string parsefile;
  size_t parse_norb = 0;
  for (int i = 1; i < argc; ++i) {
    std::string a(argv[i]);
    if (a == "--parse") parsefile = argv[++i];
    else if (a == "--norb") parse_norb = std::strtoul(argv[++i], nullptr, 10);
    else if (a == "--fcidump") fcidumpfile = argv[++i];
    else if (a == "--adetfile") adetfile = argv[++i];
    else if (a == "--bdetfile") bdetfile = argv[++i];
    else if (a == "--reps") reps = std::atoi(argv[++i]);
    else if (a == "--blocks") blocks = std::atoi(argv[++i]);
    else if (a == "--rows") rows = std::strtoul(argv[++i], nullptr, 10);
    else if (a == "--no_hii") no_hii = true;
    else if (a == "--target_s") target_s = std::atof(argv[++i]);
    else {
      std::fprintf(stderr, "ref_bench: unknown argument %s\n", a.c_str());
      return 2;
    }
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
      ts += (r ? "," : "") + std::to_string(seconds_since(p0));
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
  MPI_Comm comm = MPI_COMM_WORLD, h_comm, b_comm, t_comm, a_comm;
  sbd::TaskCommunicator(comm, 1, 1, 1, 1, h_comm, b_comm, t_comm, a_comm);
  auto t0 = std::chrono::steady_clock::now();
  std::vector<sbd::TaskHelpers> helper;
  sbd::MakeHelpers(adet, bdet, bit_length, L, helper, h_comm, b_comm, t_comm, 1, 1);
  sbd::RemakeHelpers(adet, bdet, bit_length, L, helper, h_comm, b_comm, t_comm, 1, 1);
  const double helper_s = seconds_since(t0);
  const size_t na = adet.size(), nb = bdet.size(), ndet = na * nb;
  std::vector<double> hii;
  auto t1 = std::chrono::steady_clock::now();
  if (no_hii) hii.assign(ndet, 0.0);
  else sbd::makeQChamDiagTerms(adet, bdet, bit_length, L, helper, I0, I1, I2, hii, h_comm, b_comm, t_comm);
  const double hii_s = seconds_since(t1);
  std::vector<double> win(ndet), wout(ndet);
#pragma omp parallel for
  for (size_t i = 0; i < ndet; ++i) win[i] = (double)((uint64_t(i) * 0x9E3779B97F4A7C15ull) >> 11) * 0x1p-53 - 0.5;
  std::printf("ndet=%zu na=%zu nb=%zu helper_s=%.6f hii_s=%.6f threads=%d", ndet, na, nb, helper_s,
              hii_s, omp_get_max_threads());
  auto call = [&]() {
    std::fill(wout.begin(), wout.end(), 0.0);
    auto s0 = std::chrono::steady_clock::now();
    sbd::mult(hii, win, wout, adet, bdet, bit_length, static_cast<size_t>(L), 1, 1, helper, I0, I1,
              I2, h_comm, b_comm, t_comm);
    return seconds_since(s0);
  };
  if (blocks > 0) {
    if (rows == 0 || rows > na) rows = na;
    std::vector<AlphaView> views;
    for (auto &h : helper) views.push_back(save_view(h));
    auto narrow = [&](size_t lo, size_t hi) {
      for (size_t t = 0; t < helper.size(); ++t) {
        // every 1-rank task covers all alpha bra strings; only the view of them changes
        set_view(helper[t], views[t], lo, hi);
      }
    };
    narrow(0, 0);
    const double fixed_s = call();
    if (target_s > 0.0) {
      const size_t r0 = std::max<size_t>(1, na / 200), lo = (na - r0) / 2;
      narrow(lo, lo + r0);
      const double probe_s = call();
      const double per_row = std::max(1e-7, (probe_s - fixed_s) / (double)r0);
      rows = std::min<size_t>(na, std::max<size_t>(1, (size_t)(target_s / per_row)));
      std::printf(" probe_rows=%zu probe_s=%.6f", r0, probe_s);
    }
    std::string bs, bstart, bsum;
    for (int k = 0; k < blocks; ++k) {
      const size_t lo = blocks > 1 ? (size_t)((double)k * (na - rows) / (blocks - 1)) : 0;
      narrow(lo, lo + rows);
      const double s = call();
      double cs = 0.0;  // the block's sigma rows (plus the diagonal pass over the whole vector)
      for (double x : wout) cs += x;
      char buf[64];
      std::snprintf(buf, sizeof buf, "%.17g", cs);
      bs += (k ? "," : "") + std::to_string(s);
      bstart += (k ? "," : "") + std::to_string(lo);
      bsum += (k ? "," : "") + std::string(buf);
    }
    for (size_t t = 0; t < helper.size(); ++t) restore_view(helper[t], views[t]);
    std::printf(" fixed_s=%.6f rows=%zu block_s=%s block_start=%s block_sum=%s", fixed_s, rows,
                bs.c_str(), bstart.c_str(), bsum.c_str());
  } else {
    std::string ts;
    for (int r = 0; r < reps; ++r) ts += (r ? "," : "") + std::to_string(call());
    std::printf(" sigma_s=%s", ts.c_str());
  }
  double cs = 0.0;
  for (double x : wout) cs += x;
  std::printf(" checksum=%.17g\n", cs);
  MPI_Finalize();
  return 0;
}
