// Drop-in `diag` CLI for the one-rank TPB selected-basis diagonalization on one B200.
//
// Mirrors apps/chemistry_tpb_selected_basis_diagonalization/main.cc and the flag parser of
// tpb/sbdiag.h:52-122: same flags, same stdout lines (" Davidson iteration", " Energy = ",
// " Sample-based diagonalization: ..."), same 1pRDM.txt / 2pRDM.txt files and energy
// decomposition (main.cc:196-319).  Extra flags select the arithmetic and the correction:
//   --precision fp64|mixed   --preconditioner diagonal|learned   --device N
//   --precond_params FILE    (the learned network's SBD_TPB_MLP_PARAMS FP32 values, raw)
// --loadname / --savename read and write the reference's one-rank wavefunction file
// (tpb/restart.h); --carryover_type 1/2/3 with --carryover_ratio / --carryover_threshold selects
// the carry-over strings on the GPU (tpb/sbdiag.h:690-736) and --carryover_adetfile /
// --carryover_bdetfile write them (main.cc:203-224).  Flags for parts outside this build
// (--dump_matrix_form_wf, more than one rank per communicator) are reported and rejected.
// --method 0 runs Davidson, --method 2 Lanczos (tpb/lanczos.h:167-320, its " Lanczos iteration"
// lines); the stored-Hamiltonian methods 1 and 3 are not built.
#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "sbd_tpb.h"
#include "tpb_io.h"

namespace {

[[noreturn]] void die(const std::string &msg) {
  std::cerr << "diag: " << msg << std::endl;
  std::exit(1);
}

// most strings one spin can produce for a carry-over type: the strings themselves (type 1), or
// every string and its singles, at most C(L, e) distinct ones (types 2, 3)
size_t carryover_capacity(int type, int L, const std::vector<uint64_t> &s) {
  if (type == SBD_TPB_CARRYOVER_DOMINANT || s.empty()) return s.size();
  const int e = __builtin_popcountll(s[0]);
  double binom = 1.0;
  for (int k = 1; k <= e; k++) binom = binom * (L - e + k) / k;
  return (size_t)std::min((double)s.size() * (1.0 + (double)e * (L - e)), binom + 0.5);
}

}  // namespace

int main(int argc, char **argv) {
  std::string adetfile = "alphadets.txt", bdetfile, fcidumpfile = "fcidump.txt", loadname, savename, precond_file;
  sbd_tpb_params prm;
  sbd_tpb_default_params(&prm);
  prm.verbose = 1;
  int do_shuffle = 0, method = 0, carryover_type = 0, comm_sizes = 1;
  double carryover_ratio = 0.0, carryover_threshold = 0.01;  // tpb/sbdiag.h:37-39
  std::string carryover_adetfile, carryover_bdetfile;
  size_t bit_length = 20;
  std::string unsupported;
  for (int i = 1; i < argc; i++) {
    const std::string a(argv[i]);
    auto next = [&]() -> std::string {
      if (i + 1 >= argc) die("missing value for " + a);
      return std::string(argv[++i]);
    };
    if (a == "--adetfile") adetfile = next();
    else if (a == "--bdetfile") bdetfile = next();
    else if (a == "--fcidump") fcidumpfile = next();
    else if (a == "--method") method = std::atoi(next().c_str());
    else if (a == "--iteration") prm.max_it = std::atoi(next().c_str());
    else if (a == "--block") prm.max_nb = std::atoi(next().c_str());
    else if (a == "--tolerance") prm.eps = std::atof(next().c_str());
    else if (a == "--max_time") prm.max_time = std::atof(next().c_str());
    else if (a == "--init") prm.init = std::atoi(next().c_str());
    else if (a == "--seed") prm.seed = std::strtoull(next().c_str(), nullptr, 10);
    else if (a == "--shuffle") do_shuffle = std::atoi(next().c_str());
    else if (a == "--rdm") prm.do_rdm = std::atoi(next().c_str());
    else if (a == "--bit_length") bit_length = std::strtoul(next().c_str(), nullptr, 10);
    else if (a == "--carryover_type") carryover_type = std::atoi(next().c_str());
    else if (a == "--carryover_ratio") carryover_ratio = std::atof(next().c_str());
    else if (a == "--carryover_threshold") carryover_threshold = std::atof(next().c_str());
    else if (a == "--carryover_adetfile") carryover_adetfile = next();
    else if (a == "--carryover_bdetfile") carryover_bdetfile = next();
    else if (a == "--adet_comm_size" || a == "--bdet_comm_size" || a == "--task_comm_size")
      comm_sizes *= std::atoi(next().c_str());
    else if (a == "--loadname") loadname = next();
    else if (a == "--savename") savename = next();
    else if (a == "--dump_matrix_form_wf") {
      const std::string v = next();
      if (!v.empty()) unsupported += " " + a;
    } else if (a == "--precision") {
      const std::string v = next();
      if (v == "fp64") prm.precision = SBD_TPB_FP64;
      else if (v == "mixed") prm.precision = SBD_TPB_MIXED;
      else die("--precision must be fp64 or mixed");
    } else if (a == "--preconditioner") {
      const std::string v = next();
      if (v == "diagonal") prm.preconditioner = SBD_TPB_PRECOND_DIAGONAL;
      else if (v == "learned") prm.preconditioner = SBD_TPB_PRECOND_LEARNED;
      else die("--preconditioner must be diagonal or learned");
    } else if (a == "--device") prm.device = std::atoi(next().c_str());
    else if (a == "--precond_params") precond_file = next();
    else if (a == "--use_precalculated_dets" || a == "--max_memory_gb_for_determinants" ||
             a == "--thrust_collapse_loops") next();
  }
  if (bit_length == 0 || bit_length > 64) die("--bit_length must be in [1, 64]");
  if (method != 0 && method != 2) die("only the matrix-free solvers are built: --method 0 (Davidson) or 2 (Lanczos)");
  prm.method = method;
  if (comm_sizes != 1) die("one rank on one GPU: --*_comm_size must be 1");
  if (prm.init != 0 && prm.init != 1) die("--init must be 0 (first determinant) or 1 (seeded random vector)");
  if (carryover_type < 0 || carryover_type > 3) die("--carryover_type must be 0, 1, 2 or 3");
  if (!unsupported.empty()) die("not built in this version:" + unsupported);

  std::cout.precision(16);
  tpbio::FciDump fd;
  std::string err;
  if (!tpbio::load_fcidump(fcidumpfile, fd, &err)) die(err);
  const int L = fd.norb;
  std::vector<uint64_t> adet, bdet;
  // string files (text or .bin, as LoadAlphaDets reads them) parsed, sorted and de-duplicated on
  // the GPU
  {
    sbd_tpb_handle *sh = nullptr;
    if (sbd_tpb_create(prm.device, &sh)) die(sbd_tpb_last_error());
    auto read = [&](const std::string &path, std::vector<uint64_t> &out) {
      std::ifstream f(path, std::ios::binary | std::ios::ate);
      if (!f) die("Failed to open alpha det file: " + path);
      const size_t bytes = (size_t)f.tellg();
      const bool bin = path.size() >= 4 && path.compare(path.size() - 4, 4, ".bin") == 0;
      const size_t cap = bin ? bytes / ((L + 7) / 8) : bytes / (L + 1) + 1;
      out.resize(std::max<size_t>(cap, 1));
      size_t n = 0;
      if (sbd_tpb_read_strings(sh, path.c_str(), L, out.data(), out.size(), &n)) die(sbd_tpb_last_error());
      out.resize(n);
      if (out.empty()) die("no strings in " + path);
    };
    read(adetfile, adet);
    if (bdetfile.empty()) bdet = adet;
    else read(bdetfile, bdet);
    sbd_tpb_destroy(sh);
  }
  if (do_shuffle) {
    tpbio::shuffle_strings(adet, 1729);
    tpbio::shuffle_strings(bdet, 137);
  }
  const size_t na = adet.size(), nb = bdet.size();
  std::vector<double> W(na * nb), density(2 * L);
  std::vector<double> one, two;
  if (prm.do_rdm) {
    one.resize(2 * (size_t)L * L);
    two.resize(4 * (size_t)L * L * L * L);
  }
  sbd_tpb_hamiltonian ham{L, fd.nelec, fd.core, fd.h1.data(), fd.eri_packed.data(), fd.eri_packed.size()};
  sbd_tpb_result res;
  std::memset(&res, 0, sizeof(res));
  res.ci_vector = W.data();
  res.density = density.data();
  res.one_rdm = prm.do_rdm ? one.data() : nullptr;
  res.two_rdm = prm.do_rdm ? two.data() : nullptr;
  // carry-over strings of the final vector, selected on the GPU inside the solve
  sbd_tpb_carryover co;
  std::memset(&co, 0, sizeof(co));
  std::vector<uint64_t> co_a, co_b;
  if (carryover_type != 0) {
    co.type = carryover_type;
    co.ratio = carryover_ratio;
    co.threshold = carryover_threshold;
    co_a.resize(std::max<size_t>(1, carryover_capacity(carryover_type, L, adet)));
    co_b.resize(std::max<size_t>(1, carryover_capacity(carryover_type, L, bdet)));
    co.astr = co_a.data();
    co.acap = co_a.size();
    co.bstr = co_b.data();
    co.bcap = co_b.size();
    res.carryover = &co;
  }
  // initial vector: HF determinant, or a stored wavefunction (tpb/sbdiag.h:280-296)
  std::vector<double> W0;
  if (!loadname.empty()) {
    const auto t0 = std::chrono::steady_clock::now();
    size_t matched = 0;
    if (!tpbio::load_wavefunction(loadname, L, bit_length, adet, bdet, W0, &matched, &err)) die(err);
    if (matched == 0) die("no stored amplitude matches the current strings: " + loadname);
    std::cout << " Elapsed time for init "
              << std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count() << " (sec) "
              << std::endl;
  }
  int rc = SBD_TPB_OK;
  if (prm.preconditioner == SBD_TPB_PRECOND_LEARNED) {
    // the learned network, read from a parameter file, attached to the handle of this solve
    if (precond_file.empty()) die("--preconditioner learned needs --precond_params FILE");
    std::vector<float> params(SBD_TPB_MLP_PARAMS);
    std::ifstream pf(precond_file, std::ios::binary);
    if (!pf.read(reinterpret_cast<char *>(params.data()), sizeof(float) * params.size()))
      die("cannot read " + std::to_string(SBD_TPB_MLP_PARAMS) + " FP32 values from " + precond_file);
    const auto t0 = std::chrono::steady_clock::now();
    sbd_tpb_handle *h = nullptr;
    sbd_tpb_precond *pc = nullptr;
    if (sbd_tpb_create(prm.device, &h) || sbd_tpb_set_hamiltonian(h, &ham) ||
        sbd_tpb_set_strings(h, adet.data(), na, bdet.data(), nb))
      die(sbd_tpb_last_error());
    const auto t1 = std::chrono::steady_clock::now();
    if (sbd_tpb_build_tables(h) || sbd_tpb_precond_create(prm.device, 0, &pc) ||
        sbd_tpb_precond_set_params(pc, params.data(), params.size()) || sbd_tpb_set_preconditioner(h, pc))
      die(sbd_tpb_last_error());
    res.seconds_tables = std::chrono::duration<double>(std::chrono::steady_clock::now() - t1).count();
    if (!prm.do_rdm) res.one_rdm = res.two_rdm = nullptr;
    rc = method == 2 ? sbd_tpb_lanczos(h, &prm, W0.empty() ? nullptr : W0.data(), &res)
                     : sbd_tpb_davidson(h, &prm, W0.empty() ? nullptr : W0.data(), &res);
    const std::string msg = rc == SBD_TPB_OK ? std::string() : std::string(sbd_tpb_last_error());
    sbd_tpb_destroy(h);
    sbd_tpb_precond_destroy(pc);
    res.seconds_total = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (rc != SBD_TPB_OK && rc != SBD_TPB_ERR_NOT_CONVERGED) die(msg);
  } else {
    rc = sbd_tpb_diag_from(&prm, &ham, adet.data(), na, bdet.data(), nb, W0.empty() ? nullptr : W0.data(), &res);
    if (rc != SBD_TPB_OK && rc != SBD_TPB_ERR_NOT_CONVERGED) die(sbd_tpb_last_error());
  }
  if (!savename.empty() && !tpbio::save_wavefunction(savename, L, bit_length, adet, bdet, W, &err)) die(err);
  co_a.resize(co.na);
  co_b.resize(co.nb);
  if ((carryover_type == 1 || carryover_type == 2) && carryover_ratio != 0.0) {
    std::cout << " truncated weight in carry-over for alpha-det = " << co.truncated_a << std::endl;
    std::cout << " truncated weight in carry-over for beta-det = " << co.truncated_b << std::endl;
  } else if (carryover_type == 3) {
    std::cout << " percentage of wf used in augmentation: " << co.total_weight * 100.0 << std::endl;
  }
  std::cout << " Elapsed time for helper construction " << res.seconds_tables << " (sec) " << std::endl;
  std::cout << " Elapsed time for davidson " << res.seconds_davidson << " (sec) " << std::endl;
  std::cout << " Energy = " << res.energy << std::endl;
  std::cout << " Sample-based diagonalization: Energy = " << res.energy << std::endl;
  std::cout << " Sample-based diagonalization: density = ";
  for (int i = 0; i < L; i++) std::cout << ((i == 0) ? "[" : ",") << density[2 * i] + density[2 * i + 1];
  std::cout << std::endl;
  std::cout << " Sample-based diagonalization: carryover bitstrings = [";
  for (size_t i = 0; i < std::min<size_t>(co_a.size(), 4); i++)
    std::cout << (i == 0 ? "" : ", ") << tpbio::make_string(co_a[i], L);
  if (co_a.size() > 4) std::cout << " ..., " << tpbio::make_string(co_a.back(), L);
  std::cout << "], size = " << co_a.size() << std::endl;
  // carry-over files: one string per line (main.cc:213-224)
  for (int spin = 0; spin < 2; spin++) {
    const std::string &f = spin ? carryover_bdetfile : carryover_adetfile;
    if (f.empty()) continue;
    std::ofstream os(f);
    if (!os) die("cannot write " + f);
    for (uint64_t x : spin ? co_b : co_a) os << tpbio::make_string(x, L) << "\n";
  }
  if (prm.do_rdm) {
    // 1pRDM.txt / 2pRDM.txt and the energy decomposition (main.cc:264-317)
    const size_t L2 = (size_t)L * L, L4 = L2 * L2;
    double onebody = 0.0, twobody = 0.0;
    std::ofstream o1("1pRDM.txt");
    o1.precision(16);
    for (int io = 0; io < L; io++)
      for (int jo = 0; jo < L; jo++) {
        const double g = one[io + (size_t)L * jo] + one[L2 + io + (size_t)L * jo];
        o1 << io << " " << jo << " " << g << std::endl;
        onebody += fd.h1[(size_t)io * L + jo] * g;
      }
    std::ofstream o2("2pRDM.txt");
    o2.precision(16);
    for (int io = 0; io < L; io++)
      for (int jo = 0; jo < L; jo++)
        for (int ia = 0; ia < L; ia++)
          for (int ja = 0; ja < L; ja++) {
            const size_t k = io + (size_t)L * jo + L2 * (ia + (size_t)L * ja);
            const double G = two[k] + two[L4 + k] + two[2 * L4 + k] + two[3 * L4 + k];
            o2 << io << " " << jo << " " << ia << " " << ja << " " << G << std::endl;
            twobody += 0.5 * fd.eri_packed[tpbio::packed_index(io, ia, jo, ja)] * G;
          }
    std::cout << " Zero-Body energy = " << fd.core << std::endl;
    std::cout << " One-Body energy = " << onebody << std::endl;
    std::cout << " Two-Body energy = " << twobody << std::endl;
    std::cout << " One-Body + Two-Body energy = " << onebody + twobody << std::endl;
    std::cout << " Zero-Body + One-Body + Two-Body energy = " << fd.core + onebody + twobody << std::endl;
  }
  return 0;
}
