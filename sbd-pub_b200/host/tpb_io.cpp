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

namespace {

std::string rank_file(const std::string &name) { return name + "000000"; }

size_t words_per_string(int norb, size_t bit_length) { return ((size_t)norb + bit_length - 1) / bit_length; }

void to_words(uint64_t s, int norb, size_t bit_length, std::vector<uint64_t> &w) {
  w.assign(words_per_string(norb, bit_length), 0);
  for (int p = 0; p < norb; p++)
    if ((s >> p) & 1) w[p / bit_length] |= 1ull << (p % bit_length);
}

bool from_words(const std::vector<uint64_t> &w, int norb, size_t bit_length, uint64_t *s) {
  uint64_t v = 0;
  for (size_t b = 0; b < w.size(); b++)
    for (size_t p = 0; p < bit_length; p++) {
      if (!((w[b] >> p) & 1)) continue;
      const size_t orb = b * bit_length + p;
      if (orb >= (size_t)norb || orb >= 64) return false;
      v |= 1ull << orb;
    }
  *s = v;
  return true;
}

}  // namespace

bool save_wavefunction(const std::string &name, int norb, size_t bit_length, const std::vector<uint64_t> &adet,
                       const std::vector<uint64_t> &bdet, const std::vector<double> &W, std::string *err) {
  if (bit_length == 0 || bit_length > 64 || W.size() != adet.size() * bdet.size()) {
    if (err) *err = "save_wavefunction: inconsistent sizes";
    return false;
  }
  std::ofstream out(rank_file(name), std::ios::binary);
  if (!out.is_open()) {
    if (err) *err = "failed to open output file " + rank_file(name);
    return false;
  }
  const uint64_t na = adet.size(), nb = bdet.size(), len = words_per_string(norb, bit_length);
  out.write(reinterpret_cast<const char *>(&na), 8);
  out.write(reinterpret_cast<const char *>(&nb), 8);
  out.write(reinterpret_cast<const char *>(&len), 8);
  std::vector<uint64_t> w;
  for (const auto *v : {&adet, &bdet})
    for (uint64_t s : *v) {
      to_words(s, norb, bit_length, w);
      out.write(reinterpret_cast<const char *>(w.data()), 8 * w.size());
    }
  out.write(reinterpret_cast<const char *>(W.data()), sizeof(double) * W.size());
  if (!out.good()) {
    if (err) *err = "write failed: " + rank_file(name);
    return false;
  }
  return true;
}

bool load_wavefunction(const std::string &name, int norb, size_t bit_length, const std::vector<uint64_t> &adet,
                       const std::vector<uint64_t> &bdet, std::vector<double> &W, size_t *matched,
                       std::string *err) {
  std::ifstream in(rank_file(name), std::ios::binary);
  if (!in.is_open()) {
    if (err) *err = "failed to open input file " + rank_file(name);
    return false;
  }
  uint64_t na = 0, nb = 0, len = 0;
  in.read(reinterpret_cast<char *>(&na), 8);
  in.read(reinterpret_cast<char *>(&nb), 8);
  in.read(reinterpret_cast<char *>(&len), 8);
  if (!in.good() || len == 0 || len > 64 || na > (1ull << 32) || nb > (1ull << 32)) {
    if (err) *err = "malformed wavefunction file " + rank_file(name);
    return false;
  }
  auto read_strings = [&](uint64_t count, std::vector<uint64_t> &out) {
    std::vector<uint64_t> w(len);
    out.resize(count);
    for (uint64_t i = 0; i < count; i++) {
      in.read(reinterpret_cast<char *>(w.data()), 8 * len);
      if (!in.good() || !from_words(w, norb, bit_length, &out[i])) return false;
    }
    return true;
  };
  std::vector<uint64_t> la, lb;
  if (!read_strings(na, la) || !read_strings(nb, lb)) {
    if (err) *err = "malformed strings in " + rank_file(name) + " (bit_length or norb differ?)";
    return false;
  }
  std::vector<double> lw(na * nb);
  in.read(reinterpret_cast<char *>(lw.data()), sizeof(double) * lw.size());
  if (!in.good()) {
    if (err) *err = "truncated amplitudes in " + rank_file(name);
    return false;
  }
  // positions of the stored strings among the current ones (current lists may be unsorted)
  auto index_of = [](const std::vector<uint64_t> &cur, const std::vector<uint64_t> &stored) {
    std::vector<std::pair<uint64_t, size_t>> sorted(cur.size());
    for (size_t i = 0; i < cur.size(); i++) sorted[i] = {cur[i], i};
    std::sort(sorted.begin(), sorted.end());
    std::vector<int64_t> pos(stored.size(), -1);
    for (size_t i = 0; i < stored.size(); i++) {
      auto it = std::lower_bound(sorted.begin(), sorted.end(), std::make_pair(stored[i], (size_t)0));
      if (it != sorted.end() && it->first == stored[i]) pos[i] = (int64_t)it->second;
    }
    return pos;
  };
  const std::vector<int64_t> pa = index_of(adet, la), pb = index_of(bdet, lb);
  W.assign(adet.size() * bdet.size(), 0.0);
  size_t m = 0;
  for (uint64_t i = 0; i < na; i++) {
    if (pa[i] < 0) continue;
    for (uint64_t j = 0; j < nb; j++) {
      if (pb[j] < 0) continue;
      W[(size_t)pa[i] * bdet.size() + (size_t)pb[j]] = lw[i * nb + j];
      m++;
    }
  }
  if (matched) *matched = m;
  return true;
}

}  // namespace tpbio
