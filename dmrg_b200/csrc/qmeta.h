// Host-side block-sparse metadata and the matvec task-list builder.
//
// QMeta is the metadata half of the reference's qtensor<T> (include/qtensor.h:26-31):
// per-leg sector sizes dim_[leg][sector], per-block labels sym_[block][leg] and
// per-leg fermion directions dir_[leg].  Values live elsewhere (device buffers).
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace dmrgx {

struct Group {
  int n = 2;            // Z_N fusion rule, src/useful.cpp:30; 8 labels for Z2^3
  bool z2cubed = false; // Z2 x Z2 x Z2 of the S4E build: labels 0..7 fuse by XOR,
                        // a negative label -b stands for b (src/useful.cpp:4-20)
  bool fermion = false; // parity ff when true, 0 when false (bosonic models)
  int ss(int a, int b) const {
    if (z2cubed) return a ^ (b < 0 ? -b : b);
    return (a + b + n) % n;
  }
  // Z_N: a%2 (src/useful.cpp:32); Z2^3: odd for labels 2..5 (src/useful.cpp:22-26)
  int ff(int a) const {
    if (!fermion) return 0;
    return z2cubed ? ((0x3C >> (a & 7)) & 1) : (a % 2);
  }
  // 1-2*((ff(x)*ff(y))%2): the reference's sign form, src/qtensor.cpp:1084
  int sign(int x, int y) const { return 1 - 2 * ((ff(x) * ff(y)) % 2); }
};

// group_n >= 1: Z_N; group_n == -8 (DMRGX_GROUP_Z2CUBED): Z2^3.  Returns false
// for any other value.
bool make_group(int group_n, int fermion, Group& G);

struct QMeta {
  std::vector<std::vector<int>> dims;  // dims[leg][sector]
  std::vector<int> dirs;               // dirs[leg]
  std::vector<std::vector<int>> syms;  // syms[block][leg]
  int nleg() const { return (int)dims.size(); }
  int64_t block_size(int b) const {
    int64_t s = 1;
    for (int l = 0; l < nleg(); l++) s *= dims[l][syms[b][l]];
    return s;
  }
  std::vector<int64_t> block_offsets() const;  // packed offsets, size nblk+1
  int64_t total() const;
  // parse the flat int layout of include/dmrgx.h ("meta"); returns error text or ""
  std::string parse(const int* meta);
};

// one row of the reference task list (src/qtensor.cpp:1046):
// [block, in_beg, out_beg, rows, cols, beta, alpha]
struct MapRow {
  int blk;
  int64_t in_beg, out_beg;
  int rows, cols, beta, alpha;
};

// generate_dim_sym (src/useful.cpp:151-194): the packed psi layout
void generate_dim_sym(const Group& G, const QMeta& lenv, int lnum, const QMeta& renv, int rnum,
                      int sector, std::vector<std::vector<int>>& dim,
                      std::vector<std::vector<int>>& sym);

int64_t get_dimension(const std::vector<std::vector<int>>& dim,
                      const std::vector<std::vector<int>>& sym);

// get_map (src/qtensor.cpp:997-1119) for transa='N', transb='T'.
// back=false: (dim_ret, sym_ret) are created; back=true: they are the given output layout.
// Returns "" or an error message.
std::string get_map(const Group& G, const QMeta& T, const std::vector<std::vector<int>>& dim,
                    const std::vector<std::vector<int>>& sym, int num, int beta, bool back,
                    std::vector<std::vector<int>>& dim_ret, std::vector<std::vector<int>>& sym_ret,
                    std::vector<MapRow>& rows);

}  // namespace dmrgx
