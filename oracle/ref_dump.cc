// Reference dump driver: TEST INFRASTRUCTURE ONLY.
//
// Links the reference's header-only TPB solver (sbd-pub include/sbd, compiled unchanged
// against mpi_shim/mpi.h) and writes its intermediate results for one input as raw binary
// files, so the golden fixtures under tests/golden/ come from the reference itself:
//
//   astr.u64 / bstr.u64   sorted strings (bit p = orbital p), LoadAlphaDets + sort_bitarray
//                         (basic/makedeterminants.h:160-186, framework/bit_manipulation.h:149)
//   task<T>_<kind>_{off,ket,cran}   excitation tables of the 1-rank task list built by
//                         MakeHelpers + RemakeHelpers (tpb/helper.h:710-854, 916-1226);
//                         off = CSR offsets (u64), ket = ket string index (u64), cran = labels (i32)
//   hii.f64               makeQChamDiagTerms (tpb/qcham.h:290-340)
//   sigma_in.f64 / sigma_out.f64   one application of mult (tpb/mult.h:625-881) to a seeded vector
//                         (--sigma_seed: normal deviates; --sigma_hash: the closed-form vector
//                         x_i = ((i * 0x9E3779B97F4A7C15 mod 2^64) >> 11) / 2^53 - 1/2, which a
//                         test regenerates exactly at any size without storing it)
//   davidson.txt / W.f64  Davidson (tpb/davidson.h:667-930) from the HF start (--init 0) or the
//                         seeded random start (--init 1 SEED: BasisInitVector, tpb/davidson.h:138-141,
//                         whose vector is also written as w0.f64), energy as in tpb/sbdiag.h:431-469
//   rdm1.f64 / rdm2.f64   Correlation (tpb/correlation.h:378-664)
//   lanczos.txt / W_lanczos.f64   Lanczos (tpb/lanczos.h:167-320) from the HF start: energy
//                         <W|H|W> (as tpb/sbdiag.h:431-469) and the final vector
//   co<k>_{a,b}.u64, carryover.txt   carry-over strings of W (tpb/sbdiag.h:690-736):
//                         co1 = CarryOverAdet/Bdet with the threshold (tpb/rdmat.h:63-100,
//                         190-227), co1r = the same with n_kept = ratio * size (:102-135,
//                         229-262) and its truncated weights, co2 = SinglesExtendHalfdets of co1
//                         (tpb/extend.h:186-320), co3 = SinglesExtendHalfdets(W, ..., cutoff)
//                         (tpb/extend.h:13-177) and its total weight.  co2 and co3 only when both
//                         spins hold the same number of electrons: for unequal counts the
//                         reference sizes the beta arrays from the alpha count (extend.h:85, 222,
//                         248-249), so co2 throws std::out_of_range and co3 broadcasts empty
//                         trailing strings (a null dereference in MpiBcast)
//
// Usage: ref_dump --fcidump F --adetfile A [--bdetfile B] [--bit_length 20] --out DIR
//                 [--sigma_seed S | --sigma_hash] [--davidson IT NB TOL] [--init I SEED] [--rdm] [--carryover RATIO THRESHOLD CUTOFF]
//                 [--lanczos IT NB TOL]
// The reference headers rely on their includer for these (as its app main.cc does).
#include <chrono>
#include <cmath>
#include <deque>
#include <unistd.h>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <random>
#include <string>
#include <vector>

#include "mpi.h"
#include "sbd/sbd.h"

namespace {

template <typename T>
void write_raw(const std::string &path, const T *p, size_t n) {
  std::FILE *f = std::fopen(path.c_str(), "wb");
  if (!f) {
    std::perror(path.c_str());
    std::exit(2);
  }
  if (n) std::fwrite(p, sizeof(T), n, f);
  std::fclose(f);
}

std::vector<uint64_t> pack_strings(const std::vector<std::vector<size_t>> &dets, size_t bit_length,
                                   int L) {
  std::vector<uint64_t> out(dets.size(), 0);
  for (size_t i = 0; i < dets.size(); ++i) {
    for (int p = 0; p < L; ++p) {
      if ((dets[i][p / bit_length] >> (p % bit_length)) & 1) out[i] |= uint64_t(1) << p;
    }
  }
  return out;
}

void dump_table(const std::string &prefix, size_t nrows, const size_t *len, size_t *const *ket,
                int *const *cran, int labels_per_entry) {
  std::vector<uint64_t> off(nrows + 1, 0);
  std::vector<uint64_t> k;
  std::vector<int32_t> c;
  for (size_t i = 0; i < nrows; ++i) {
    off[i + 1] = off[i] + len[i];
    for (size_t j = 0; j < len[i]; ++j) {
      k.push_back(ket[i][j]);
      for (int l = 0; l < labels_per_entry; ++l) c.push_back(cran[i][labels_per_entry * j + l]);
    }
  }
  write_raw(prefix + "_off.u64", off.data(), off.size());
  write_raw(prefix + "_ket.u64", k.data(), k.size());
  write_raw(prefix + "_cran.i32", c.data(), c.size());
}

}  // namespace

int main(int argc, char **argv) {
  std::string fcidumpfile, adetfile, bdetfile, out = ".";
  size_t bit_length = 20;
  long sigma_seed = -1;
  bool sigma_hash = false;
  int dav_it = 0, dav_nb = 0, dav_init = 0;
  unsigned long long dav_seed = 1729;
  double dav_tol = 1e-8;
  bool do_rdm = false;
  double co_ratio = -1.0, co_threshold = 0.0, co_cutoff = 0.0;
  int lz_it = 0, lz_nb = 0;
  double lz_tol = 1e-8;
  for (int i = 1; i < argc; ++i) {
    std::string a(argv[i]);
    if (a == "--fcidump") fcidumpfile = argv[++i];
    else if (a == "--adetfile") adetfile = argv[++i];
    else if (a == "--bdetfile") bdetfile = argv[++i];
    else if (a == "--bit_length") bit_length = std::atoi(argv[++i]);
    else if (a == "--out") out = argv[++i];
    else if (a == "--sigma_seed") sigma_seed = std::atol(argv[++i]);
    else if (a == "--sigma_hash") sigma_hash = true;
    else if (a == "--davidson") {
      dav_it = std::atoi(argv[++i]);
      dav_nb = std::atoi(argv[++i]);
      dav_tol = std::atof(argv[++i]);
    } else if (a == "--init") {
      dav_init = std::atoi(argv[++i]);
      dav_seed = std::strtoull(argv[++i], nullptr, 10);
    } else if (a == "--rdm") do_rdm = true;
    else if (a == "--lanczos") {
      lz_it = std::atoi(argv[++i]);
      lz_nb = std::atoi(argv[++i]);
      lz_tol = std::atof(argv[++i]);
    } else if (a == "--carryover") {
      co_ratio = std::atof(argv[++i]);
      co_threshold = std::atof(argv[++i]);
      co_cutoff = std::atof(argv[++i]);
    }
  }
  int provided;
  MPI_Init_thread(&argc, &argv, MPI_THREAD_FUNNELED, &provided);
  MPI_Comm comm = MPI_COMM_WORLD;

  sbd::FCIDump fcidump = sbd::LoadFCIDump(fcidumpfile);
  int L = 0, N = 0;
  double I0 = 0.0;
  sbd::oneInt<double> I1;
  sbd::twoInt<double> I2;
  sbd::SetupIntegrals(fcidump, L, N, I0, I1, I2);

  std::vector<std::vector<size_t>> adet, bdet;
  sbd::LoadAlphaDets(adetfile, adet, bit_length, L);
  sbd::sort_bitarray(adet);
  if (bdetfile.empty()) {
    bdet = adet;
  } else {
    sbd::LoadAlphaDets(bdetfile, bdet, bit_length, L);
    sbd::sort_bitarray(bdet);
  }
  auto a64 = pack_strings(adet, bit_length, L);
  auto b64 = pack_strings(bdet, bit_length, L);
  write_raw(out + "/astr.u64", a64.data(), a64.size());
  write_raw(out + "/bstr.u64", b64.data(), b64.size());

  MPI_Comm h_comm, b_comm, t_comm, a_comm;
  sbd::TaskCommunicator(comm, 1, 1, 1, 1, h_comm, b_comm, t_comm, a_comm);
  std::vector<sbd::TaskHelpers> helper;
  sbd::MakeHelpers(adet, bdet, bit_length, L, helper, h_comm, b_comm, t_comm, 1, 1);
  sbd::RemakeHelpers(adet, bdet, bit_length, L, helper, h_comm, b_comm, t_comm, 1, 1);

  {
    std::ofstream ofs(out + "/tasks.txt");
    for (size_t t = 0; t < helper.size(); ++t) {
      const auto &h = helper[t];
      ofs << t << " " << h.taskType << " " << h.braAlphaStart << " " << h.braAlphaEnd << " "
          << h.braBetaStart << " " << h.braBetaEnd << " " << h.ketAlphaStart << " "
          << h.ketAlphaEnd << " " << h.ketBetaStart << " " << h.ketBetaEnd << "\n";
      const size_t na = h.braAlphaEnd - h.braAlphaStart;
      const size_t nb = h.braBetaEnd - h.braBetaStart;
      const std::string p = out + "/task" + std::to_string(t);
      if (h.taskType != 1) {
        dump_table(p + "_sa", na, h.SinglesFromAlphaLen, h.SinglesFromAlphaSM.data(),
                   h.SinglesAlphaCrAnSM.data(), 2);
      }
      if (h.taskType == 2) {
        dump_table(p + "_da", na, h.DoublesFromAlphaLen, h.DoublesFromAlphaSM.data(),
                   h.DoublesAlphaCrAnSM.data(), 4);
      }
      if (h.taskType != 2) {
        dump_table(p + "_sb", nb, h.SinglesFromBetaLen, h.SinglesFromBetaSM.data(),
                   h.SinglesBetaCrAnSM.data(), 2);
      }
      if (h.taskType == 1) {
        dump_table(p + "_db", nb, h.DoublesFromBetaLen, h.DoublesFromBetaSM.data(),
                   h.DoublesBetaCrAnSM.data(), 4);
      }
    }
  }

  std::vector<double> hii;
  sbd::makeQChamDiagTerms(adet, bdet, bit_length, L, helper, I0, I1, I2, hii, h_comm, b_comm,
                          t_comm);
  write_raw(out + "/hii.f64", hii.data(), hii.size());

  if (sigma_seed >= 0 || sigma_hash) {
    std::vector<double> win(hii.size()), wout(hii.size(), 0.0);
    if (sigma_hash) {
      for (size_t i = 0; i < win.size(); ++i)
        win[i] = (double)((uint64_t(i) * 0x9E3779B97F4A7C15ull) >> 11) * 0x1p-53 - 0.5;
    } else {
      std::mt19937_64 g(static_cast<uint64_t>(sigma_seed));
      std::normal_distribution<double> nd(0.0, 1.0);
      for (auto &x : win) x = nd(g);
    }
    sbd::mult(hii, win, wout, adet, bdet, bit_length, static_cast<size_t>(L), 1, 1, helper, I0,
              I1, I2, h_comm, b_comm, t_comm);
    write_raw(out + "/sigma_in.f64", win.data(), win.size());
    write_raw(out + "/sigma_out.f64", wout.data(), wout.size());
  }

  if (dav_it > 0) {
    std::vector<double> W;
    sbd::BasisInitVector(W, adet, bdet, 1, 1, h_comm, b_comm, t_comm, dav_init, dav_seed);
    if (dav_init != 0) write_raw(out + "/w0.f64", W.data(), W.size());
    sbd::Davidson(hii, W, adet, bdet, bit_length, static_cast<size_t>(L), 1, 1, helper, I0, I1, I2,
                  h_comm, b_comm, t_comm, dav_it, dav_nb, dav_tol, 86400.0);
    std::vector<double> C(W.size(), 0.0);
    sbd::mult(hii, W, C, adet, bdet, bit_length, static_cast<size_t>(L), 1, 1, helper, I0, I1, I2,
              h_comm, b_comm, t_comm);
    double E = 0.0;
    sbd::InnerProduct(W, C, E, b_comm);
    std::ofstream ofs(out + "/davidson.txt");
    ofs.precision(17);
    ofs << E << "\n";
    write_raw(out + "/W.f64", W.data(), W.size());
    if (do_rdm) {
      std::vector<std::vector<double>> one, two;
      sbd::Correlation(W, adet, bdet, bit_length, static_cast<size_t>(L), 1, 1, helper, h_comm,
                       b_comm, t_comm, one, two);
      std::vector<double> r1, r2;
      for (auto &v : one) r1.insert(r1.end(), v.begin(), v.end());
      for (auto &v : two) r2.insert(r2.end(), v.begin(), v.end());
      write_raw(out + "/rdm1.f64", r1.data(), r1.size());
      write_raw(out + "/rdm2.f64", r2.data(), r2.size());
    }
    if (co_ratio >= 0.0) {
      auto dump = [&](const std::string &name, const std::vector<std::vector<size_t>> &d) {
        auto p = pack_strings(d, bit_length, L);
        write_raw(out + "/" + name + ".u64", p.data(), p.size());
      };
      std::vector<std::vector<size_t>> co_a, co_b, ex_a, ex_b;
      sbd::CarryOverAdet(W, adet, bdet, 1, 1, b_comm, co_a, co_threshold);
      sbd::CarryOverBdet(W, adet, bdet, 1, 1, b_comm, co_b, co_threshold);
      dump("co1_a", co_a);
      dump("co1_b", co_b);
      const bool same_count = sbd::bitcount(adet[0], bit_length, L) == sbd::bitcount(bdet[0], bit_length, L);
      if (same_count) {
        sbd::SinglesExtendHalfdets(co_a, co_b, bit_length, static_cast<size_t>(L), 1, 1, b_comm, ex_a, ex_b);
        dump("co2_a", ex_a);
        dump("co2_b", ex_b);
      }
      double tw_a = 0.0, tw_b = 0.0, total = 0.0;
      std::vector<std::vector<size_t>> cr_a, cr_b;
      sbd::CarryOverAdet(W, adet, bdet, 1, 1, b_comm, static_cast<size_t>(co_ratio * adet.size()), cr_a, tw_a);
      sbd::CarryOverBdet(W, adet, bdet, 1, 1, b_comm, static_cast<size_t>(co_ratio * bdet.size()), cr_b, tw_b);
      dump("co1r_a", cr_a);
      dump("co1r_b", cr_b);
      if (same_count) {
        std::vector<std::vector<size_t>> c3_a, c3_b;
        sbd::SinglesExtendHalfdets(W, adet, bdet, bit_length, static_cast<size_t>(L), 1, 1, b_comm,
                                   co_cutoff, c3_a, c3_b, total);
        dump("co3_a", c3_a);
        dump("co3_b", c3_b);
      }
      std::ofstream oc(out + "/carryover.txt");
      oc.precision(17);
      oc << co_ratio << " " << co_threshold << " " << co_cutoff << " " << tw_a << " " << tw_b << " " << total << "\n";
    }
  }
  if (lz_it > 0) {
    std::vector<double> W;
    sbd::BasisInitVector(W, adet, bdet, 1, 1, h_comm, b_comm, t_comm, 0, 1729);
    sbd::Lanczos(hii, W, adet, bdet, bit_length, static_cast<size_t>(L), 1, 1, helper, I0, I1, I2,
                 h_comm, b_comm, t_comm, lz_it, lz_nb, lz_tol);
    std::vector<double> C(W.size(), 0.0);
    sbd::mult(hii, W, C, adet, bdet, bit_length, static_cast<size_t>(L), 1, 1, helper, I0, I1, I2,
              h_comm, b_comm, t_comm);
    double E = 0.0;
    sbd::InnerProduct(W, C, E, b_comm);
    std::ofstream ofs(out + "/lanczos.txt");
    ofs.precision(17);
    ofs << E << "\n";
    write_raw(out + "/W_lanczos.f64", W.data(), W.size());
  }
  MPI_Finalize();
  return 0;
}
