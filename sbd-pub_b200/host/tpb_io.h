// Host-side input parsing for the drop-in `diag` CLI: FCIDUMP and alpha/beta string files.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace tpbio {

struct FciDump {
  int norb = 0;
  int nelec = 0;
  int ms2 = 0;
  double core = 0.0;
  std::vector<double> h1;          // norb*norb, row-major, symmetric
  std::vector<double> eri_packed;  // 8-fold packed store (basic/integrals.h:64-107)
};

// FCIDUMP text as framework/fcidump.h:29-141 reads it and basic/makeintegrals.h:123-174 stores
// it.  Returns false with *err set on failure.
bool load_fcidump(const std::string &path, FciDump &out, std::string *err);

// Text form of a string as sbd::makestring prints it (orbital norb-1 first).
std::string make_string(uint64_t s, int norb);

// Reference's ShuffleDet (basic/determinants.h:622-628): keep entry 0, shuffle the rest with
// std::mt19937(seed).
void shuffle_strings(std::vector<uint64_t> &s, unsigned int seed);

size_t packed_index(int i, int j, int k, int l);

// Wavefunction file of one rank as tpb/restart.h:19-68 writes it (file name = name + "000000"):
// adet count, bdet count and words per string (size_t each), the strings as words of
// bit_length bits (bit p of a string in word p / bit_length, bit p % bit_length, as
// bit_manipulation.h:215-230 builds them), then W (double, index Ia*nb + Ib, reference sign
// convention).
bool save_wavefunction(const std::string &name, int norb, size_t bit_length, const std::vector<uint64_t> &adet,
                       const std::vector<uint64_t> &bdet, const std::vector<double> &W, std::string *err);
// Reads such a file and places each stored amplitude on the current strings (tpb/restart.h:70+,
// one rank): W[ia*nb + ib] for every stored pair whose strings are both present, zero elsewhere.
// *matched receives how many stored amplitudes found a place.
bool load_wavefunction(const std::string &name, int norb, size_t bit_length, const std::vector<uint64_t> &adet,
                       const std::vector<uint64_t> &bdet, std::vector<double> &W, size_t *matched,
                       std::string *err);

}  // namespace tpbio
