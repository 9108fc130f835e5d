// sbd_tpb_sbd.hpp -- drop-in binding of libsbdtpb for the reference's TPB application (C++17,
// header-only).
//
// This is the code a maintainer of ncsa/sbd-pub adds to run its TPB selected-basis
// diagonalization on one B200: include it after the reference's "sbd/sbd.h" (it uses sbd's own
// types and its restart-file functions) and replace the call
//     sbd::tpb::diag(comm, sbd_data, fcidump, adet, bdet, loadname, savename, energy, density,
//                    co_adet, co_bdet, one_p_rdm, two_p_rdm);
// of apps/chemistry_tpb_selected_basis_diagonalization/main.cc:190 by sbd_b200::diag with the same
// arguments.  It accepts what sbd::tpb::diag (tpb/sbdiag.h:139-151) accepts on one MPI rank with
// --method 0 or 2, and fills the same outputs: the energy <W|H|W>, the orbital occupations
// density[2p+s], the carry-over strings (tpb/sbdiag.h:690-736), and with do_rdm the spin-resolved
// 1/2-RDMs in the layouts of tpb/correlation.h:378-664.  --loadname / --savename go through the
// reference's own LoadWavefunction / SaveWavefunction (tpb/restart.h:21-66, 415; called as
// tpb/sbdiag.h:288 and :743 call them).  Errors of the library become std::runtime_error with its
// message, as the reference reports failures by exceptions.
#pragma once

#include <algorithm>
#include <stdexcept>
#include <string>
#include <vector>

#include "sbd_tpb.h"

namespace sbd_b200 {

// Strings as sbd holds them (bit_length bits per size_t word, bit p = orbital p) <-> uint64.
inline std::vector<uint64_t> pack_strings(const std::vector<std::vector<size_t>> &d, size_t bl, int L) {
  std::vector<uint64_t> o(d.size(), 0);
  for (size_t i = 0; i < d.size(); ++i)
    for (int p = 0; p < L; ++p)
      if ((d[i][p / bl] >> (p % bl)) & 1) o[i] |= uint64_t(1) << p;
  return o;
}

inline std::vector<std::vector<size_t>> unpack_strings(const std::vector<uint64_t> &o, size_t bl, int L) {
  std::vector<std::vector<size_t>> d(o.size(), std::vector<size_t>((L + bl - 1) / bl, 0));
  for (size_t i = 0; i < o.size(); ++i)
    for (int p = 0; p < L; ++p)
      if ((o[i] >> p) & 1) d[i][p / bl] |= size_t(1) << (p % bl);
  return d;
}

inline void check(int rc) {
  if (rc != SBD_TPB_OK && rc != SBD_TPB_ERR_NOT_CONVERGED) throw std::runtime_error(sbd_tpb_last_error());
}

inline void diag(const MPI_Comm &comm, const sbd::tpb::SBD &s, const sbd::FCIDump &fcidump,
                 const std::vector<std::vector<size_t>> &adet, const std::vector<std::vector<size_t>> &bdet,
                 const std::string &loadname, const std::string &savename, double &energy,
                 std::vector<double> &density, std::vector<std::vector<size_t>> &co_adet,
                 std::vector<std::vector<size_t>> &co_bdet, std::vector<std::vector<double>> &one_p_rdm,
                 std::vector<std::vector<double>> &two_p_rdm, int device = 0) {
  int nrank = 1;
  MPI_Comm_size(comm, &nrank);
  if (nrank != 1 || s.adet_comm_size != 1 || s.bdet_comm_size != 1 || s.task_comm_size != 1 || s.h_comm_size != 1)
    throw std::runtime_error("sbd_b200::diag runs one rank on one GPU");
  if (s.method != SBD_TPB_METHOD_DAVIDSON && s.method != SBD_TPB_METHOD_LANCZOS)
    throw std::runtime_error("sbd_b200::diag: --method 0 (Davidson) or 2 (Lanczos) only");
  if (s.init != 0 && s.init != 1) throw std::runtime_error("sbd_b200::diag: --init 0 or 1 only");

  // the Hamiltonian as SetupIntegrals builds it (framework/makeintegrals.h:123-174): I1 over spin
  // orbitals (the alpha block is the spatial matrix), I2 as the 8-fold packed store
  int L = 0, N = 0;
  double I0 = 0.0;
  sbd::oneInt<double> I1;
  sbd::twoInt<double> I2;
  sbd::SetupIntegrals(fcidump, L, N, I0, I1, I2);
  std::vector<double> h1((size_t)L * L);
  for (int i = 0; i < L; ++i)
    for (int j = 0; j < L; ++j) h1[(size_t)i * L + j] = I1.Value(2 * i, 2 * j);
  const sbd_tpb_hamiltonian ham{L, N, I0, h1.data(), I2.store.data(), I2.store.size()};

  sbd_tpb_params p;
  sbd_tpb_default_params(&p);
  p.max_it = s.max_it;
  p.max_nb = s.max_nb;
  p.eps = s.eps;
  p.max_time = s.max_time;
  p.init = s.init;
  p.seed = s.seed;
  p.do_rdm = s.do_rdm;
  p.method = s.method;
  p.device = device;

  const auto a = pack_strings(adet, s.bit_length, L), b = pack_strings(bdet, s.bit_length, L);
  const size_t ndet = a.size() * b.size();

  // start vector: the reference's restart file when asked for (W in the reference's order and sign
  // convention, as sbd_tpb_diag_from takes it), else the start --init selects (HF determinant or
  // the seeded random vector, both built by the library)
  MPI_Comm h_comm, b_comm, t_comm, a_comm;
  sbd::TaskCommunicator(comm, 1, 1, 1, 1, h_comm, b_comm, t_comm, a_comm);
  std::vector<double> W0;
  if (!loadname.empty()) {
    sbd::LoadWavefunction(loadname, adet, bdet, 1, 1, h_comm, b_comm, t_comm, W0);
    if (W0.size() != ndet) throw std::runtime_error("sbd_b200::diag: loaded wavefunction has the wrong size");
  }

  density.assign(2 * (size_t)L, 0.0);
  std::vector<double> one(s.do_rdm ? 2 * (size_t)L * L : 0), two(s.do_rdm ? 4 * (size_t)L * L * L * L : 0);
  std::vector<double> W(savename.empty() ? 0 : ndet);
  sbd_tpb_result r{};
  r.density = density.data();
  r.one_rdm = s.do_rdm ? one.data() : nullptr;
  r.two_rdm = s.do_rdm ? two.data() : nullptr;
  r.ci_vector = savename.empty() ? nullptr : W.data();

  // carry-over strings: type 1 keeps at most n strings per spin, types 2 and 3 at most
  // n * (1 + e (L - e)) (each string and its singles), never more than C(L, e)
  sbd_tpb_carryover co{};
  co.type = s.carryover_type;
  co.ratio = s.ratio;
  co.threshold = s.threshold;
  std::vector<uint64_t> ca, cb;
  if (co.type != SBD_TPB_CARRYOVER_NONE) {
    auto cap = [&](const std::vector<uint64_t> &v) {
      const int e = __builtin_popcountll(v[0]);
      double c = 1.0;
      for (int k = 1; k <= e; ++k) c = c * (L - e + k) / k;
      return co.type == SBD_TPB_CARRYOVER_DOMINANT
                 ? v.size()
                 : (size_t)std::min((double)v.size() * (1.0 + e * (L - e)), c + 0.5);
    };
    ca.resize(cap(a));
    cb.resize(cap(b));
    co.astr = ca.data();
    co.acap = ca.size();
    co.bstr = cb.data();
    co.bcap = cb.size();
    r.carryover = &co;
  }
  if (loadname.empty()) check(sbd_tpb_diag(&p, &ham, a.data(), a.size(), b.data(), b.size(), &r));
  else check(sbd_tpb_diag_from(&p, &ham, a.data(), a.size(), b.data(), b.size(), W0.data(), &r));
  energy = r.energy;
  if (co.type != SBD_TPB_CARRYOVER_NONE) {
    ca.resize(co.na);
    cb.resize(co.nb);
    co_adet = unpack_strings(ca, s.bit_length, L);
    co_bdet = unpack_strings(cb, s.bit_length, L);
  }
  if (s.do_rdm) {  // onebody[s][i + L*j], twobody[s + 2t][...]
    const size_t L2 = (size_t)L * L, L4 = L2 * L2;
    one_p_rdm.assign(2, std::vector<double>());
    for (int k = 0; k < 2; ++k) one_p_rdm[k].assign(one.begin() + k * L2, one.begin() + (k + 1) * L2);
    two_p_rdm.assign(4, std::vector<double>());
    for (int k = 0; k < 4; ++k) two_p_rdm[k].assign(two.begin() + k * L4, two.begin() + (k + 1) * L4);
  }
  if (!savename.empty()) sbd::SaveWavefunction(savename, adet, bdet, 1, 1, h_comm, b_comm, t_comm, W);
}

}  // namespace sbd_b200
