// Host-side input parsing for the drop-in `diag` CLI (see tpb_io.h).
#include "tpb_io.h"

#include <algorithm>
#include <fstream>
#include <map>
#include <random>
#include <sstream>

namespace tpbio {

size_t packed_index(int I, int J, int K, int L) {
  const int mij = std::max(I, J), nij = std::min(I, J);
  const int mkl = std::max(K, L), nkl = std::min(K, L);
  const size_t ij = (size_t)mij * (mij + 1) / 2 + nij;
  const size_t kl = (size_t)mkl * (mkl + 1) / 2 + nkl;
  const size_t a = std::max(ij, kl), b = std::min(ij, kl);
  return a * (a + 1) / 2 + b;
}

static std::string trim(const std::string &s) {
  const size_t a = s.find_first_not_of(" \t");
  if (a == std::string::npos) return std::string();
  const size_t b = s.find_last_not_of(" \t");
  return s.substr(a, b - a + 1);
}

bool load_fcidump(const std::string &path, FciDump &out, std::string *err) {
  std::ifstream in(path);
  if (!in.is_open()) {
    if (err) *err = "Failed to open FCIDUMP file: " + path;
    return false;
  }
  std::string line, header;
  bool in_header = true;
  struct Entry {
    double v;
    int i, j, k, l;
  };
  std::vector<Entry> ints;
  while (std::getline(in, line)) {
    if (!line.empty() && line.back() == '\r') line.pop_back();
    if (line.empty() || line[0] == '!') continue;
    if (in_header) {
      if (line.find("&END") != std::string::npos) {
        in_header = false;
        continue;
      }
      const size_t p = line.find("&FCI");
      if (p != std::string::npos) line.erase(p, 4);
      header += line;
    } else {
      std::stringstream ss(line);
      Entry e;
      if (ss >> e.v >> e.i >> e.j >> e.k >> e.l) ints.push_back(e);
    }
  }
  std::map<std::string, std::string> kv;
  std::stringstream hs(header);
  std::string tok;
  while (std::getline(hs, tok, ',')) {
    const size_t eq = tok.find('=');
    if (eq == std::string::npos) continue;
    kv[trim(tok.substr(0, eq))] = trim(tok.substr(eq + 1));
  }
  if (!kv.count("NORB")) {
    if (err) *err = "FCIDUMP header has no NORB";
    return false;
  }
  out.norb = std::atoi(kv["NORB"].c_str());
  out.nelec = kv.count("NELEC") ? std::atoi(kv["NELEC"].c_str()) : 0;
  out.ms2 = kv.count("MS2") ? std::atoi(kv["MS2"].c_str()) : 0;
  const int L = out.norb;
  if (L < 1 || L > 64) {
    if (err) *err = "NORB must be in [1, 64] (strings are held in one 64-bit word)";
    return false;
  }
  const size_t B = (size_t)L * (L + 1) / 2;
  out.h1.assign((size_t)L * L, 0.0);
  out.eri_packed.assign(B * (B + 1) / 2, 0.0);
  out.core = 0.0;
  for (const Entry &e : ints) {
    if (e.i == 0 && e.j == 0 && e.k == 0 && e.l == 0) {
      out.core = e.v;
    } else if (e.k == 0 && e.l == 0) {
      if (e.i < 1 || e.j < 1 || e.i > L || e.j > L) {
        if (err) *err = "FCIDUMP one-electron index out of range";
        return false;
      }
      out.h1[(size_t)(e.i - 1) * L + (e.j - 1)] = e.v;
      out.h1[(size_t)(e.j - 1) * L + (e.i - 1)] = e.v;
    } else {
      if (e.i < 1 || e.j < 1 || e.k < 1 || e.l < 1 || e.i > L || e.j > L || e.k > L || e.l > L) {
        if (err) *err = "FCIDUMP two-electron index out of range";
        return false;
      }
      out.eri_packed[packed_index(e.i - 1, e.j - 1, e.k - 1, e.l - 1)] = e.v;
    }
  }
  return true;
}

bool load_strings(const std::string &path, int norb, std::vector<uint64_t> &out, std::string *err) {
  std::ifstream in(path);
  if (!in.is_open()) {
    if (err) *err = "Failed to open alpha det file: " + path;
    return false;
  }
  if (path.size() >= 4 && path.substr(path.size() - 4) == ".bin") {
    if (err) *err = "binary string files are not supported; use the .txt form";
    return false;
  }
  out.clear();
  std::string line;
  while (std::getline(in, line)) {
    while (!line.empty() && (line.back() == '\r' || line.back() == ' ')) line.pop_back();
    if (line.empty()) continue;
    if ((int)line.size() < norb) {
      if (err) *err = "string shorter than NORB: '" + line + "'";
      return false;
    }
    uint64_t v = 0;
    for (int i = 0; i < norb; i++) {
      const char c = line[norb - 1 - i];
      if (c == '1') v |= 1ull << i;
      else if (c != '0') {
        if (err) *err = "string with characters other than 0/1: '" + line + "'";
        return false;
      }
    }
    out.push_back(v);
  }
  std::sort(out.begin(), out.end());
  out.erase(std::unique(out.begin(), out.end()), out.end());
  return true;
}

std::string make_string(uint64_t s, int norb) {
  std::string r(norb, '0');
  for (int i = 0; i < norb; i++)
    if ((s >> i) & 1) r[norb - 1 - i] = '1';
  return r;
}

void shuffle_strings(std::vector<uint64_t> &s, unsigned int seed) {
  if (s.size() <= 1) return;
  std::mt19937 g(seed);
  std::shuffle(s.begin() + 1, s.end(), g);
}

}  // namespace tpbio
