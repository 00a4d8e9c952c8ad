// The in-place LP standard form (build_plain_lp_into, used by the batched path) against the general
// builder (build_std_form): bit-exact on random LPs with shifts, upper bounds, Le/Ge/Eq rows,
// maximisation, scaling on and off, and the plain-column test on columns with zeros.
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>

#include "stdform.hpp"

using namespace sov;

int main() {
  std::mt19937 rng(7);
  int bad = 0, tested = 0, nonplain = 0;
  for (int t = 0; t < 3000; ++t) {
    const int m = 1 + rng() % 40, n = 1 + rng() % 80;
    std::vector<int> cp(1, 0), ri;
    std::vector<double> v, c(n), lb(n), ub(n), rhs(m);
    std::vector<int8_t> sense(m);
    for (int j = 0; j < n; ++j) {
      for (int r = 0; r < m; ++r)
        if (rng() % 4 == 0) {
          ri.push_back(r);
          v.push_back((int(rng() % 2001) - 1000) / 37.0);
        }
      if (t % 50 == 0 && !ri.empty() && rng() % 3 == 0) v.back() = 0.0;  // a zero: not plain
      cp.push_back(static_cast<int>(ri.size()));
      c[j] = (int(rng() % 200) - 100) / 3.0;
      lb[j] = (rng() % 3 == 0) ? (int(rng() % 100) - 50) / 7.0 : 0.0;
      ub[j] = (rng() % 3 == 0) ? lb[j] + (rng() % 100) / 3.0 : 1e30;
    }
    for (int r = 0; r < m; ++r) {
      rhs[r] = (int(rng() % 1000) - 500) / 11.0;
      sense[r] = static_cast<int8_t>(rng() % 3);
    }
    sov_model p{};
    p.n = n;
    p.m = m;
    p.maximize = static_cast<int32_t>(rng() % 2);
    p.col_ptr = cp.data();
    p.row_idx = ri.data();
    p.values = v.data();
    p.obj = c.data();
    p.lb = lb.data();
    p.ub = ub.data();
    p.sense = sense.data();
    p.rhs = rhs.data();
    for (int sc = 0; sc < 2; ++sc) {
      const StdForm f = build_std_form(p, false, sc != 0);
      LpShape s;
      if (!plain_lp_shape(p, &s)) {
        ++nonplain;
        continue;
      }
      ++tested;
      if (s.m != f.m || s.n != f.n || s.nnz != f.nnz()) {
        ++bad;
        continue;
      }
      std::vector<int> cpo(s.n + 1), rio(s.nnz), rpo(s.m + 1), cio(s.nnz);
      std::vector<double> vo(s.nnz), rvo(s.nnz), bo(s.m), co(s.n), sho(s.n_struct), cso(s.n), rso(s.m);
      const LpFormOut o{cpo.data(), rio.data(), vo.data(), rpo.data(), cio.data(), rvo.data(),
                        bo.data(),  co.data(),  sho.data(), cso.data(), rso.data()};
      LpFormInfo info{};
      build_plain_lp_into(p, s, sc != 0, o, &info);
      auto eqd = [](const std::vector<double>& a, const std::vector<double>& b) {
        return a.size() == b.size() && std::memcmp(a.data(), b.data(), 8 * a.size()) == 0;
      };
      const bool ok = cpo == f.col_ptr && rio == f.row_idx && eqd(vo, f.val) && rpo == f.row_ptr &&
                      cio == f.col_idx && eqd(rvo, f.rval) && eqd(bo, f.b) && eqd(co, f.c) && eqd(sho, f.shift) &&
                      eqd(cso, f.col_scale) && eqd(rso, f.row_scale) && info.scaling_applied == f.scaling_applied &&
                      info.coef_min_before == f.coef_min_before && info.coef_max_before == f.coef_max_before &&
                      info.coef_min_after == f.coef_min_after && info.coef_max_after == f.coef_max_after;
      if (!ok) {
        ++bad;
        if (bad < 5) std::printf("mismatch t=%d scaling=%d\n", t, sc);
      }
    }
  }
  std::printf("tested %d, non-plain %d, mismatches %d\n", tested, nonplain, bad);
  return bad != 0 || tested < 1000 || nonplain == 0;
}
