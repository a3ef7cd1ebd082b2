// Sector bookkeeping of the matvec: psi layout and task lists.
// Integer work only; results must equal the reference's bit for bit.
#include "qmeta.h"

#include <unordered_map>

namespace dmrgx {

std::vector<int64_t> QMeta::block_offsets() const {
  std::vector<int64_t> off(syms.size() + 1, 0);
  for (size_t b = 0; b < syms.size(); b++) off[b + 1] = off[b] + block_size((int)b);
  return off;
}

int64_t QMeta::total() const { return block_offsets().back(); }

std::string QMeta::parse(const int* meta) {
  if (!meta) return "null metadata";
  int k = 0;
  int nl = meta[k++];
  int nb = meta[k++];
  if (nl <= 0 || nl > 16 || nb < 0) return "bad leg/block count in metadata";
  dims.assign(nl, {});
  std::vector<int> nsec(nl);
  for (int l = 0; l < nl; l++) {
    nsec[l] = meta[k++];
    if (nsec[l] <= 0 || nsec[l] > 4096) return "bad sector count in metadata";
  }
  for (int l = 0; l < nl; l++) {
    dims[l].resize(nsec[l]);
    for (int s = 0; s < nsec[l]; s++) {
      dims[l][s] = meta[k++];
      if (dims[l][s] < 0) return "negative sector size in metadata";
    }
  }
  dirs.resize(nl);
  for (int l = 0; l < nl; l++) dirs[l] = meta[k++];
  syms.assign(nb, std::vector<int>(nl));
  for (int b = 0; b < nb; b++)
    for (int l = 0; l < nl; l++) {
      int s = meta[k++];
      if (s < 0 || s >= nsec[l]) return "block label out of range in metadata";
      syms[b][l] = s;
    }
  return "";
}

// all label tuples of the given radices in lexicographic order (src/useful.cpp:119-134)
static std::vector<std::vector<int>> label_tuples(const std::vector<int>& radix) {
  std::vector<std::vector<int>> out;
  int64_t total = 1;
  for (int r : radix) total *= r;
  out.reserve((size_t)total);
  std::vector<int> cur(radix.size(), 0);
  for (int64_t i = 0; i < total; i++) {
    out.push_back(cur);
    for (int p = (int)radix.size() - 1; p >= 0; p--) {
      if (++cur[p] < radix[p]) break;
      cur[p] = 0;
    }
  }
  return out;
}

bool make_group(int group_n, int fermion, Group& G) {
  G = Group();
  G.fermion = fermion != 0;
  if (group_n == -8) {
    G.n = 8;
    G.z2cubed = true;
    return true;
  }
  if (group_n < 1 || group_n > 4096) return false;
  G.n = group_n;
  return true;
}

void generate_dim_sym(const Group& G, const QMeta& lenv, int lnum, const QMeta& renv, int rnum,
                      int sector, std::vector<std::vector<int>>& dim,
                      std::vector<std::vector<int>>& sym) {
  dim.clear();
  for (int i = 0; i < lnum; i++) dim.push_back(lenv.dims[lenv.nleg() - lnum + i]);
  for (int i = 0; i < rnum; i++) dim.push_back(renv.dims[renv.nleg() - rnum + i]);
  std::vector<int> lr, rr;
  for (int i = 0; i < lnum; i++) lr.push_back((int)dim[i].size());
  for (int i = 0; i < rnum; i++) rr.push_back((int)dim[lnum + i].size());
  auto lt = label_tuples(lr), rt = label_tuples(rr);
  std::vector<int> lsum(lt.size()), rsum(rt.size());
  for (size_t i = 0; i < lt.size(); i++) {
    int s = 0;
    for (int x : lt[i]) s = G.ss(s, x);
    lsum[i] = s;
  }
  for (size_t i = 0; i < rt.size(); i++) {
    int s = 0;
    for (int x : rt[i]) s = G.ss(s, x);
    rsum[i] = s;
  }
  sym.clear();
  if (sector == -1) {
    sym.push_back(std::vector<int>(dim.size(), 0));
    return;
  }
  // the reference's order (src/useful.cpp:172-188): left charge s = 0..N-1, then
  // left tuples, then right tuples, each lexicographic.  The tuples are bucketed
  // by their charge (order kept within a bucket) instead of rescanning every
  // pair for every s, which is N |lt| |rt| work (33 M pairs for U(1) in Z_32).
  std::unordered_map<int, std::vector<int>> lby, rby;
  for (size_t l = 0; l < lt.size(); l++) lby[lsum[l]].push_back((int)l);
  for (size_t r = 0; r < rt.size(); r++) rby[rsum[r]].push_back((int)r);
  size_t count = 0;
  for (int s = 0; s < G.n; s++) {
    auto li = lby.find(s), ri = rby.find(G.ss(sector, -s));
    if (li != lby.end() && ri != rby.end()) count += li->second.size() * ri->second.size();
  }
  sym.reserve(count);
  for (int s = 0; s < G.n; s++) {
    const int t = G.ss(sector, -s);
    auto li = lby.find(s), ri = rby.find(t);
    if (li == lby.end() || ri == rby.end()) continue;
    for (int l : li->second)
      for (int r : ri->second) {
        std::vector<int> v = lt[l];
        v.insert(v.end(), rt[r].begin(), rt[r].end());
        sym.push_back(std::move(v));
      }
  }
}

int64_t get_dimension(const std::vector<std::vector<int>>& dim,
                      const std::vector<std::vector<int>>& sym) {
  int64_t d = 0;
  for (auto& s : sym) {
    int64_t t = 1;
    for (size_t j = 0; j < dim.size(); j++) t *= dim[j][s[j]];
    d += t;
  }
  return d;
}

// A linear key of a label tuple (the reference's `loc`, src/qtensor.cpp:1092-1093).
static int64_t label_key(const std::vector<int>& st, const std::vector<std::vector<int>>& dim) {
  int64_t loc = 0;
  for (size_t q = 0; q < dim.size(); q++) loc = loc * (int64_t)dim[q].size() + st[q];
  return loc;
}

std::string get_map(const Group& G, const QMeta& T, const std::vector<std::vector<int>>& dim,
                    const std::vector<std::vector<int>>& sym, int num, int beta, bool back,
                    std::vector<std::vector<int>>& dim_ret, std::vector<std::vector<int>>& sym_ret,
                    std::vector<MapRow>& rows) {
  const int nT = T.nleg();
  const int indexa = nT - num;                    // transa = 'N'
  const int indexb = (int)dim.size() - num;       // transb = 'T'
  if (num <= 0 || indexa < 0 || indexb < 0) return "get_map: bad contraction count";
  for (int i = 0; i < num; i++)
    if (T.dims[indexa + i] != dim[indexb + i]) return "get_map: contracted dimensions differ";

  std::vector<std::vector<int>> new_dim_ret;
  for (int i = 0; i < nT; i++)
    if (i < indexa || i >= indexa + num) new_dim_ret.push_back(T.dims[i]);
  for (int i = 0; i < (int)dim.size(); i++)
    if (i < indexb || i >= indexb + num) new_dim_ret.push_back(dim[i]);

  // per input block: total size, row size, begin offset (src/qtensor.cpp:1031-1041)
  const size_t nin = sym.size();
  std::vector<int64_t> tot(nin), rowsz(nin), beg(nin);
  int64_t acc = 0;
  for (size_t i = 0; i < nin; i++) {
    int64_t t = 1, r = 1;
    for (size_t s = 0; s < dim.size(); s++) t *= dim[s][sym[i][s]];
    if (indexb)
      for (int s = 0; s < indexb; s++) r *= dim[s][sym[i][s]];
    else
      for (int s = 0; s < num; s++) r *= dim[s][sym[i][s]];
    tot[i] = t;
    rowsz[i] = r;
    beg[i] = acc;
    acc += t;
  }

  rows.clear();
  std::unordered_map<int64_t, int> key2out;  // label key -> output block index
  std::vector<int64_t> out_off;              // output block offsets
  std::vector<char> first;
  if (back) {
    out_off.assign(sym_ret.size(), 0);
    for (size_t i = 0; i < sym_ret.size(); i++) {
      key2out[label_key(sym_ret[i], dim_ret)] = (int)i;
      if (i + 1 < sym_ret.size()) {
        int64_t d = 1;
        for (size_t j = 0; j < dim_ret.size(); j++) d *= dim_ret[j][sym_ret[i][j]];
        out_off[i + 1] = out_off[i] + d;
      }
    }
    first.assign(sym_ret.size(), 1);
  } else {
    dim_ret = new_dim_ret;
    sym_ret.clear();
  }
  int64_t next_off = 0;  // end of the created layout (back=false)

  // match on contracted labels: index the input blocks by their contracted tuple
  std::unordered_map<int64_t, std::vector<int>> in_by_key;
  for (size_t j = 0; j < nin; j++) {
    int64_t key = 0;
    for (int k = 0; k < num; k++) key = key * 4099 + sym[j][indexb + k];
    in_by_key[key].push_back((int)j);
  }
  std::vector<int> st(dim_ret.size());
  for (size_t i = 0; i < T.syms.size(); i++) {
    const auto& ts = T.syms[i];
    int64_t key = 0;
    for (int k = 0; k < num; k++) key = key * 4099 + ts[indexa + k];
    auto it = in_by_key.find(key);
    if (it == in_by_key.end()) continue;
    int d_b = 0;
    if (!back)
      for (int k = 0; k < nT; k++) d_b = G.ss(d_b, ts[k] * T.dirs[k]);
    for (int j : it->second) {
      bool match = true;  // guard against key collisions
      for (int k = 0; k < num; k++)
        if (ts[indexa + k] != sym[j][indexb + k]) match = false;
      if (!match || tot[j] == 0) continue;
      MapRow row;
      row.blk = (int)i;
      row.in_beg = beg[j];
      row.rows = (int)rowsz[j];
      row.cols = (int)(tot[j] / rowsz[j]);
      row.beta = beta;
      row.alpha = 1;
      if (!back) {
        int a_p = 0;
        for (int k = 0; k < (int)dim.size() - num; k++) a_p = G.ss(a_p, sym[j][k]);
        row.alpha = G.sign(d_b, a_p);
      }
      int ad = 0;
      for (int k = 0; k < nT; k++)
        if (k < indexa || k >= indexa + num) st[ad++] = ts[k];
      for (int k = 0; k < (int)dim.size(); k++)
        if (k < indexb || k >= indexb + num) st[ad++] = sym[j][k];
      int64_t loc = label_key(st, dim_ret);
      auto f = key2out.find(loc);
      if (f != key2out.end()) {
        int t = f->second;
        row.out_beg = out_off[t];
        if (back && first[t])
          first[t] = 0;
        else
          row.beta = 1;
        rows.push_back(row);
      } else if (!back) {
        int64_t d = 1;
        for (size_t q = 0; q < dim_ret.size(); q++) d *= dim_ret[q][st[q]];
        key2out[loc] = (int)sym_ret.size();
        out_off.push_back(next_off);
        row.out_beg = next_off;
        next_off += d;
        sym_ret.push_back(st);
        rows.push_back(row);
      }
    }
  }
  return "";
}

}  // namespace dmrgx
