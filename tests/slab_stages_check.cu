// Host check of the batched guard folds (ctca_b200/csrc/slab.cuh): for every
// combination of periodic / open field axes and both array kinds, the stages
// of slab_stages keep the list order, hold pairwise independent operations,
// and give the same array as the operations one after the other, whatever
// the order inside a stage.  Built and run by tests/test_slab_stages.py.
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>

#include "slab.cuh"

using namespace emsesg;

static int64_t count_of(const SlabOp& o) {
  const int ax = o.axis, ea = ax == 0 ? 1 : 0, eb = ax == 2 ? 1 : 2;
  return (int64_t)o.depth * (o.hi[ea] - o.lo[ea] + 1) * (o.hi[eb] - o.lo[eb] + 1) * o.nc;
}

static void apply(std::vector<long long>& a, const FieldDesc& f, const SlabOp& o) {
  SlabArgs s;
  s.o = o;
  s.f = f;
  s.count = count_of(o);
  for (int64_t t = 0; t < s.count; t++) slab_apply(a.data(), s, t);
}

int main() {
  int bad = 0, cases = 0, launches_seq = 0, launches_st = 0;
  std::mt19937_64 rng(7);
  const int dims[][3] = {{5, 6, 7}, {8, 8, 8}, {16, 12, 9}};
  for (const auto& n : dims)
    for (int fb = 0; fb < 8; fb++)
      for (int kind = 0; kind < 2; kind++) {
        emsesg_config c{};
        c.nx = n[0];
        c.ny = n[1];
        c.nz = n[2];
        for (int d = 0; d < 3; d++) c.nfbnd[d] = (fb >> d) & 1;
        const int ncomp = kind == 0 ? 1 : 3;
        const std::vector<SlabOp> ops = fold_ops(c, kind, ncomp);
        const auto st = slab_stages(ops);
        // a generous array around every plane the operations touch
        FieldDesc f{ncomp, -6, n[0] + 13, n[1] + 13, n[2] + 13};
        std::vector<long long> a0((size_t)f.size());
        for (auto& v : a0) v = (long long)(rng() % 2000001) - 1000000;
        std::vector<long long> seq = a0, fwd = a0, rev = a0;
        for (const SlabOp& o : ops) apply(seq, f, o);
        size_t k = 0;
        for (const auto& s : st) {
          for (size_t i = 0; i < s.size(); i++) {
            for (int e = 0; e < 3; e++)
              if (e != s[i].axis && (s[i].lo[e] != ops[k].lo[e] || s[i].hi[e] != ops[k].hi[e])) bad++;
            if (s[i].op != ops[k].op || s[i].axis != ops[k].axis || s[i].dst0 != ops[k].dst0 ||
                s[i].src0 != ops[k].src0 || s[i].c0 != ops[k].c0)
              bad++;  // order kept
            k++;
            for (size_t j = 0; j < i; j++)
              if (!slab_independent(s[i], s[j])) bad++;
          }
          for (size_t i = 0; i < s.size(); i++) apply(fwd, f, s[i]);
          for (size_t i = s.size(); i-- > 0;) apply(rev, f, s[i]);
        }
        if (k != ops.size() || fwd != seq || rev != seq) {
          bad++;
          std::printf("mismatch n=%dx%dx%d nfbnd=%d kind=%d\n", n[0], n[1], n[2], fb, kind);
        }
        cases++;
        launches_seq += (int)ops.size();
        launches_st += (int)st.size();
      }
  std::printf("%s cases=%d ops=%d stages=%d\n", bad ? "FAIL" : "ok", cases, launches_seq, launches_st);
  return bad ? 1 : 0;
}
