// Component-split CG product kernels for large product graphs (see
// cg_codegen.h, generate_cg_split_source).
//
// The energy of a saved SUS2-SH graph is a sum over terminal scalar rows,
// E = sum_rows w sum_terms c V[a] V[b] (the site-energy fusion of
// gpu_sh_forward_energy_backward_compact_rows, src/force/sus2_sh.cu:5674-5778,
// 5893-5905), and in every standard graph of body order <= 5 each
// intermediate moment feeds terminal rows only.  Such "local" intermediates,
// linked by the terminal terms that multiply two of them, fall apart into
// small connected components: for the real-CG graph one component per
// (coupled rank L, component M), because the rank-0 coupling of two rank-L
// tensors pairs equal M only.  A component is evaluated on its own --
// values, adjoints, energy and the back-propagation into the basic moments --
// with every value a register, so the straight-line code of the whole graph
// never holds more than one component live.  The basic moments ("globals")
// and their adjoints live in lane-private shared memory ([slot][block]);
// intermediates that feed non-terminal rows (body 6) join the globals and
// are computed before and back-propagated after the components.  Every
// component, and every chunk of global work, is its own __noinline__
// function, which keeps ptxas time linear in the graph size.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <map>
#include <numeric>
#include <set>
#include <sstream>

#include "cg_codegen.h"

namespace sus2sh {
namespace {

std::string lit(double c, bool f32) {
  char buf[64];
  if (f32) std::snprintf(buf, sizeof(buf), "%.9ef", static_cast<double>(static_cast<float>(c)));
  else std::snprintf(buf, sizeof(buf), "%.17e", c);
  return buf;
}

unsigned long long fnv1a(const std::string& s) {
  unsigned long long h = 1469598103934665603ull;
  for (unsigned char ch : s) {
    h ^= ch;
    h *= 1099511628211ull;
  }
  return h;
}

struct Term {
  int a, b;  // moments
  double w;  // coefficient x row weight
};

enum Cls : char { kDead, kBasic, kLocal, kShared, kTerminal };

struct Component {
  std::vector<int> locals;  // moments, in row order
  std::vector<Term> terms;  // terminal terms with at least one local operand
};

// The terms of a row grouped by the magnitude of their coefficient as the
// working precision rounds it (in order of first appearance), with each
// term's sign.
struct MagGroup {
  double magnitude;
  std::vector<size_t> terms;
  std::vector<bool> negative;
};

std::vector<MagGroup> magnitude_groups(const Row& row, bool use_float) {
  std::vector<MagGroup> out;
  std::map<double, size_t> index;
  for (size_t t = 0; t < row.coeff.size(); ++t) {
    double c = row.coeff[t];
    if (use_float) c = static_cast<double>(static_cast<float>(c));
    const double m = std::fabs(c);
    auto it = index.find(m);
    if (it == index.end()) {
      it = index.emplace(m, out.size()).first;
      out.push_back({m, {}, {}});
    }
    out[it->second].terms.push_back(t);
    out[it->second].negative.push_back(c < 0.0);
  }
  return out;
}

}  // namespace

bool generate_cg_split_source(const HostModel& m, const Layered& lay, bool use_float,
                              const std::vector<int>& basic_canon, int ncanon, CgSource* out,
                              std::string* why) {
  const int M = m.moments, Bb = m.basic_count;
  const char* T = use_float ? "float" : "double";
  const char* FMA = use_float ? "fmaf" : "fma";
  const std::string zero = use_float ? "0.0f" : "0.0";
  const std::string half = use_float ? "0.5f" : "0.5";
  auto fail = [&](const std::string& s) {
    if (why) *why = s;
    return false;
  };

  std::vector<int> row_of(M, -1);
  for (size_t r = 0; r < lay.rows.size(); ++r) row_of[lay.rows[r].target] = static_cast<int>(r);
  std::vector<double> weight(M, 0.0);
  std::vector<char> is_scalar(M, 0);
  for (int s = 0; s < m.scalar_count; ++s) {
    weight[m.moment_mapping[s]] += m.moment_coeffs[s];
    is_scalar[m.moment_mapping[s]] = 1;
  }
  // liveness: rows are sorted by layer, so a backward walk sees consumers first
  std::vector<char> live(M, 0);
  for (int x = 0; x < M; ++x)
    if (is_scalar[x] && weight[x] != 0.0) live[x] = 1;
  for (int r = static_cast<int>(lay.rows.size()) - 1; r >= 0; --r) {
    const Row& row = lay.rows[r];
    if (!live[row.target]) continue;
    for (size_t t = 0; t < row.left.size(); ++t) live[row.left[t]] = live[row.right[t]] = 1;
  }
  // classes
  std::vector<Cls> cls(M, kDead);
  std::vector<std::vector<int>> cons(M);  // live consumer rows (unique)
  for (size_t r = 0; r < lay.rows.size(); ++r) {
    const Row& row = lay.rows[r];
    if (!live[row.target]) continue;
    std::set<int> ops(row.left.begin(), row.left.end());
    ops.insert(row.right.begin(), row.right.end());
    for (int o : ops) cons[o].push_back(static_cast<int>(r));
  }
  for (int x = 0; x < M; ++x) {
    if (x < Bb) {
      cls[x] = kBasic;
      continue;
    }
    if (row_of[x] < 0 || !live[x]) continue;
    if (lay.terminal[x]) {
      cls[x] = kTerminal;
      continue;
    }
    bool all_terminal = !cons[x].empty();
    for (int r : cons[x]) all_terminal = all_terminal && lay.terminal[lay.rows[r].target];
    cls[x] = all_terminal ? kLocal : kShared;
  }
  // global slots: basics, then shared intermediates in row order
  std::vector<int> gslot(M, -1);
  int nglob = 0;
  for (int b = 0; b < Bb; ++b) gslot[b] = nglob++;
  std::vector<int> shared_rows;
  for (size_t r = 0; r < lay.rows.size(); ++r)
    if (cls[lay.rows[r].target] == kShared) {
      gslot[lay.rows[r].target] = nglob++;
      shared_rows.push_back(static_cast<int>(r));
    }
  // union-find over locals joined by terminal terms
  std::vector<int> parent(M);
  std::iota(parent.begin(), parent.end(), 0);
  std::function<int(int)> find = [&](int x) {
    while (parent[x] != x) x = parent[x] = parent[parent[x]];
    return x;
  };
  std::vector<Term> gterms;  // terminal terms between two globals
  std::vector<Term> all_terms;
  for (const Row& row : lay.rows) {
    if (cls[row.target] != kTerminal) continue;
    const double w = weight[row.target];
    for (size_t t = 0; t < row.left.size(); ++t) {
      const int a = row.left[t], b = row.right[t];
      if (cls[a] == kDead || cls[b] == kDead || cls[a] == kTerminal || cls[b] == kTerminal)
        return fail("terminal row reads a moment the split kernel cannot place");
      all_terms.push_back({a, b, row.coeff[t] * w});
      if (cls[a] == kLocal && cls[b] == kLocal) parent[find(a)] = find(b);
    }
  }
  std::map<int, int> comp_of_root;
  std::vector<Component> comps;
  for (const Row& row : lay.rows) {
    const int x = row.target;
    if (cls[x] != kLocal) continue;
    const int root = find(x);
    auto it = comp_of_root.find(root);
    if (it == comp_of_root.end()) {
      it = comp_of_root.emplace(root, static_cast<int>(comps.size())).first;
      comps.emplace_back();
    }
    comps[it->second].locals.push_back(x);
  }
  for (const Term& t : all_terms) {
    const int x = cls[t.a] == kLocal ? t.a : (cls[t.b] == kLocal ? t.b : -1);
    if (x < 0) gterms.push_back(t);
    else comps[comp_of_root[find(x)]].terms.push_back(t);
  }
  size_t max_locals = 0;
  for (const Component& c : comps) max_locals = std::max(max_locals, c.locals.size());
  constexpr size_t kMaxLocals = 160;
  if (max_locals > kMaxLocals)
    return fail("largest component has " + std::to_string(max_locals) + " values (limit " +
                std::to_string(kMaxLocals) + ")");
  // launch shape: lane-private globals + adjoints in shared memory; two CTAs
  // per SM where they fit.  The program is megabytes of straight-line code
  // whose instruction fetch bounds the kernel; warps that run it in step
  // share the fetched lines (measured on the l4k4 body-5 graph: rotating the
  // function order per warp, so that their misses overlap, ran 4-8x slower).
  const size_t esz = use_float ? 4 : 8;
  int block = 0, min_blocks = 1;
  for (int want_ctas : {2, 1}) {
    for (int b : {128, 64, 32}) {
      if (2ull * nglob * b * esz * want_ctas <= 227ull * 1024 - 1024ull * want_ctas) {
        block = b;
        min_blocks = want_ctas;
        break;
      }
    }
    if (block) break;
  }
  if (!block) return fail("basic moments and shared intermediates do not fit shared memory");
  const std::string BLK = std::to_string(block);

  std::vector<std::string> fn_defs, fn_decls;  // device functions
  std::string sig;                             // signature of the function being emitted
  auto add_fn = [&](const std::string& signature, const std::string& def) {
    fn_decls.push_back("extern \"C\" __device__ " + signature + ";\n");
    fn_defs.push_back(def);
  };
  std::ostringstream pre_calls, post_calls;  // kernel body calls before / after the energy functions
  std::vector<std::string> energy_fns;           // components and global-term chunks (any order)
  long long terms_emitted = 0;
  int nfunc = 0;
  auto sv = [&](int slot) { return "sv[" + std::to_string(slot) + " * " + BLK + "]"; };
  auto sa = [&](int slot) { return "sa[" + std::to_string(slot) + " * " + BLK + "]"; };

  // ---- shared intermediates: values (row order), chunked
  {
    std::ostringstream f;
    int in_chunk = 0;
    auto open = [&]() {
      f.str("");
      sig = std::string("void s") + std::to_string(nfunc) + "(" + T + "* __restrict__ sv)";
      f << "extern \"C\" __device__ __noinline__ " << sig << " {\n";
    };
    auto close = [&]() {
      f << "}\n";
      add_fn(sig, f.str());
      pre_calls << "  s" << nfunc << "(sv);\n";
      ++nfunc;
      in_chunk = 0;
    };
    bool opened = false;
    for (int r : shared_rows) {
      if (!opened) {
        open();
        opened = true;
      }
      const Row& row = lay.rows[r];
      f << "  { " << T << " v = " << zero << ";\n";
      for (size_t t = 0; t < row.left.size(); ++t)
        f << "    v = " << FMA << "(" << lit(row.coeff[t], use_float) << " * " << sv(gslot[row.left[t]]) << ", "
          << sv(gslot[row.right[t]]) << ", v);\n";
      f << "    " << sv(gslot[row.target]) << " = v; }\n";
      terms_emitted += static_cast<long long>(row.left.size());
      in_chunk += static_cast<int>(row.left.size());
      if (in_chunk >= 1500) {
        close();
        opened = false;
      }
    }
    if (opened) close();
  }

  // ---- components
  for (const Component& c : comps) {
    std::ostringstream f;
    sig = std::string(T) + " c" + std::to_string(nfunc) + "(const " + T + "* __restrict__ sv, " + T +
          "* __restrict__ sa)";
    f << "extern \"C\" __device__ __noinline__ " << sig << " {\n  " << T << " e = " << zero << ";\n";
    std::map<int, int> pos;
    for (size_t i = 0; i < c.locals.size(); ++i) pos[c.locals[i]] = static_cast<int>(i);
    std::vector<Term> terms = c.terms;
    auto tkey = [&](const Term& t) {
      int k = -1;
      if (cls[t.a] == kLocal) k = std::max(k, pos[t.a]);
      if (cls[t.b] == kLocal) k = std::max(k, pos[t.b]);
      return k;
    };
    std::stable_sort(terms.begin(), terms.end(), [&](const Term& x, const Term& y) { return tkey(x) < tkey(y); });
    std::vector<int> last_term(c.locals.size(), -1);
    for (size_t i = 0; i < terms.size(); ++i) {
      if (cls[terms[i].a] == kLocal) last_term[pos[terms[i].a]] = static_cast<int>(i);
      if (cls[terms[i].b] == kLocal) last_term[pos[terms[i].b]] = static_cast<int>(i);
    }
    // event list: -1-i = finalize local i, i >= 0 = term i
    std::vector<int> events;
    for (size_t i = 0; i < c.locals.size(); ++i)
      if (last_term[i] < 0) events.push_back(-1 - static_cast<int>(i));
    for (size_t i = 0; i < terms.size(); ++i) {
      events.push_back(static_cast<int>(i));
      for (size_t j = 0; j < c.locals.size(); ++j)
        if (last_term[j] == static_cast<int>(i)) events.push_back(-1 - static_cast<int>(j));
    }
    // last event touching each global accumulator
    std::map<int, int> last_acc;
    for (size_t e = 0; e < events.size(); ++e) {
      const int ev = events[e];
      if (ev >= 0) {
        const Term& t = terms[ev];
        if (cls[t.a] != kLocal) last_acc[t.a] = static_cast<int>(e);
        if (cls[t.b] != kLocal) last_acc[t.b] = static_cast<int>(e);
      } else {
        const Row& row = lay.rows[row_of[c.locals[-1 - ev]]];
        for (size_t t = 0; t < row.left.size(); ++t) last_acc[row.left[t]] = last_acc[row.right[t]] = static_cast<int>(e);
      }
    }
    std::map<int, std::vector<int>> flush_at;
    for (auto& kv : last_acc) flush_at[kv.second].push_back(kv.first);
    std::set<int> loaded, have_v, have_h, have_k, have_q;
    auto g = [&](int x) {  // global value (lazy load)
      if (!loaded.count(x)) {
        f << "  const " << T << " g" << x << " = " << sv(gslot[x]) << ";\n";
        loaded.insert(x);
      }
      return "g" + std::to_string(x);
    };
    auto val = [&](int x) -> std::string {  // value of local or global
      if (cls[x] != kLocal) return g(x);
      if (!have_v.count(x)) {
        // v = sum_t c_t a_t b_t as sum over the row's coefficient magnitudes m of
        // m * (sum of +-a_t b_t): one multiply-add per term and one per
        // magnitude (real-CG rows repeat magnitudes) instead of two per term
        const Row& row = lay.rows[row_of[x]];
        const std::vector<MagGroup> groups = magnitude_groups(row, use_float);
        const std::string xs = std::to_string(x);
        for (size_t gi = 0; gi < groups.size(); ++gi) {
          const std::string sn = "s" + xs + "_" + std::to_string(gi);
          const MagGroup& gr = groups[gi];
          for (size_t k = 0; k < gr.terms.size(); ++k) {
            const size_t t = gr.terms[k];
            const std::string la = (gr.negative[k] ? "-" : "") + g(row.left[t]), rb = g(row.right[t]);
            if (k == 0) f << "  " << T << " " << sn << " = " << la << " * " << rb << ";\n";
            else f << "  " << sn << " = " << FMA << "(" << la << ", " << rb << ", " << sn << ");\n";
          }
          if (gi == 0) f << "  " << T << " v" << xs << " = " << lit(gr.magnitude, use_float) << " * " << sn << ";\n";
          else f << "  v" << xs << " = " << FMA << "(" << lit(gr.magnitude, use_float) << ", " << sn << ", v" << xs
                 << ");\n";
        }
        terms_emitted += static_cast<long long>(row.left.size());
        have_v.insert(x);
      }
      return "v" + std::to_string(x);
    };
    // accumulators of local values (h, k) start with their first product; those
    // of globals (q) start from the global's adjoint in shared memory, so the
    // flush at the global's last use in the component is a single store
    auto acc = [&](std::set<int>& have, const char* pfx, int x, const std::string& a, const std::string& b) {
      const std::string nm = pfx + std::to_string(x);
      if (!have.count(x)) {
        if (&have == &have_q)
          f << "  " << T << " " << nm << " = " << FMA << "(" << a << ", " << b << ", " << sa(gslot[x]) << ");\n";
        else
          f << "  " << T << " " << nm << " = " << a << " * " << b << ";\n";
        have.insert(x);
      } else {
        f << "  " << nm << " = " << FMA << "(" << a << ", " << b << ", " << nm << ");\n";
      }
    };
    for (size_t e = 0; e < events.size(); ++e) {
      const int ev = events[e];
      if (ev >= 0) {
        const Term& t = terms[ev];
        const bool la = cls[t.a] == kLocal, lb = cls[t.b] == kLocal;
        if (la && lb) {
          if (t.a == t.b) {
            acc(have_h, "h", t.a, lit(2.0 * t.w, use_float), val(t.a));
          } else {
            const std::string va = val(t.a), vb = val(t.b);
            acc(have_h, "h", t.a, lit(t.w, use_float), vb);
            acc(have_h, "h", t.b, lit(t.w, use_float), va);
          }
          terms_emitted += 2;
        } else {
          const int x = la ? t.a : t.b, y = la ? t.b : t.a;
          const std::string vx = val(x), gy = g(y);
          acc(have_k, "k", x, lit(t.w, use_float), gy);
          acc(have_q, "q", y, lit(t.w, use_float), vx);
          terms_emitted += 2;
        }
      } else {
        const int x = c.locals[-1 - ev];
        const std::string vx = val(x);
        const std::string xs = std::to_string(x);
        const double seed = weight[x];
        const bool h = have_h.count(x) > 0, k = have_k.count(x) > 0;
        std::string kx;
        if (k && seed != 0.0) kx = "(k" + xs + " + " + lit(seed, use_float) + ")";
        else if (k) kx = "k" + xs;
        else if (seed != 0.0) kx = lit(seed, use_float);
        const std::string gx = "gx" + xs;
        if (h && !kx.empty()) {
          f << "  const " << T << " " << gx << " = h" << xs << " + " << kx << ";\n";
          f << "  e = " << FMA << "(" << vx << ", " << FMA << "(" << half << ", h" << xs << ", " << kx << "), e);\n";
        } else if (h) {
          f << "  const " << T << " " << gx << " = h" << xs << ";\n";
          f << "  e = " << FMA << "(" << half << " * " << vx << ", " << gx << ", e);\n";
        } else if (!kx.empty()) {
          f << "  const " << T << " " << gx << " = " << kx << ";\n";
          f << "  e = " << FMA << "(" << vx << ", " << gx << ", e);\n";
        }
        // back-propagation through the row of x into the global accumulators
        // (a local without any adjoint contributes nothing)
        if (h || !kx.empty()) {
          // one product m * gx per coefficient magnitude of the row, then two
          // multiply-adds per term with the term's sign on the operand
          const Row& row = lay.rows[row_of[x]];
          const std::vector<MagGroup> groups = magnitude_groups(row, use_float);
          for (size_t gi = 0; gi < groups.size(); ++gi) {
            const MagGroup& gr = groups[gi];
            const std::string pn = "p" + xs + "_" + std::to_string(gi);
            f << "  const " << T << " " << pn << " = " << lit(gr.magnitude, use_float) << " * " << gx << ";\n";
            for (size_t k = 0; k < gr.terms.size(); ++k) {
              const size_t t = gr.terms[k];
              const int a = row.left[t], b = row.right[t];
              const std::string ps = gr.negative[k] ? "(-" + pn + ")" : pn;
              acc(have_q, "q", a, ps, g(b));
              acc(have_q, "q", b, ps, g(a));
            }
          }
          terms_emitted += 2 * static_cast<long long>(row.left.size());
        }
      }
      auto fl = flush_at.find(static_cast<int>(e));
      if (fl != flush_at.end())
        for (int y : fl->second)
          if (have_q.count(y)) f << "  " << sa(gslot[y]) << " = q" << y << ";\n";
    }
    f << "  return e;\n}\n";
    add_fn(sig, f.str());
    energy_fns.push_back("c" + std::to_string(nfunc));
    ++nfunc;
  }
  // ---- terminal terms between two globals and seeds of global scalars, chunked
  {
    std::vector<int> seeds;
    for (int x = 0; x < M; ++x)
      if ((cls[x] == kBasic || cls[x] == kShared) && is_scalar[x] && weight[x] != 0.0) seeds.push_back(x);
    size_t ti = 0, si = 0;
    while (ti < gterms.size() || si < seeds.size()) {
      std::ostringstream f;
      std::set<int> loaded, have_q;
      auto g = [&](int x) {
        if (!loaded.count(x)) {
          f << "  const " << T << " g" << x << " = " << sv(gslot[x]) << ";\n";
          loaded.insert(x);
        }
        return "g" + std::to_string(x);
      };
      auto accq = [&](int x, const std::string& a, const std::string& b) {
        const std::string nm = "q" + std::to_string(x);
        if (!have_q.count(x)) {
          f << "  " << T << " " << nm << " = " << a << " * " << b << ";\n";
          have_q.insert(x);
        } else {
          f << "  " << nm << " = " << FMA << "(" << a << ", " << b << ", " << nm << ");\n";
        }
      };
      sig = std::string(T) + " t" + std::to_string(nfunc) + "(const " + T + "* __restrict__ sv, " + T +
            "* __restrict__ sa)";
      f << "extern \"C\" __device__ __noinline__ " << sig << " {\n  " << T << " e = " << zero << ";\n";
      int n = 0;
      for (; si < seeds.size() && n < 1500; ++si, ++n) {
        const int x = seeds[si];
        const std::string w = lit(weight[x], use_float);
        const std::string gx = g(x);
        f << "  e = " << FMA << "(" << w << ", " << gx << ", e);\n";
        if (!have_q.count(x)) {
          f << "  " << T << " q" << x << " = " << w << ";\n";
          have_q.insert(x);
        } else {
          f << "  q" << x << " += " << w << ";\n";
        }
      }
      for (; ti < gterms.size() && n < 1500; ++ti, ++n) {
        const Term& t = gterms[ti];
        const std::string ga = g(t.a), gb = g(t.b), w = lit(t.w, use_float);
        const std::string pn = "pt" + std::to_string(ti);
        f << "  const " << T << " " << pn << " = " << w << " * " << ga << ";\n";
        f << "  e = " << FMA << "(" << pn << ", " << gb << ", e);\n";
        if (!have_q.count(t.b)) {
          f << "  " << T << " q" << t.b << " = " << pn << ";\n";
          have_q.insert(t.b);
        } else {
          f << "  q" << t.b << " += " << pn << ";\n";
        }
        accq(t.a, w, gb);
        terms_emitted += 3;
      }
      for (int x : have_q) f << "  " << sa(gslot[x]) << " += q" << x << ";\n";
      f << "  return e;\n}\n";
      add_fn(sig, f.str());
      energy_fns.push_back("t" + std::to_string(nfunc));
      ++nfunc;
    }
  }

  // ---- shared intermediates: back-propagation in reverse row order, chunked
  {
    std::ostringstream f;
    bool opened = false;
    int in_chunk = 0;
    for (auto it = shared_rows.rbegin(); it != shared_rows.rend(); ++it) {
      if (!opened) {
        f.str("");
        sig = std::string("void b") + std::to_string(nfunc) + "(const " + T + "* __restrict__ sv, " + T + "* sa)";
        f << "extern \"C\" __device__ __noinline__ " << sig << " {\n";
        opened = true;
      }
      const Row& row = lay.rows[*it];
      f << "  { const " << T << " gx = " << sa(gslot[row.target]) << ";\n";
      for (size_t t = 0; t < row.left.size(); ++t) {
        const int a = gslot[row.left[t]], b = gslot[row.right[t]];
        f << "    { const " << T << " q = " << lit(row.coeff[t], use_float) << " * gx;\n";
        f << "      " << sa(a) << " = " << FMA << "(q, " << sv(b) << ", " << sa(a) << ");\n";
        f << "      " << sa(b) << " = " << FMA << "(q, " << sv(a) << ", " << sa(b) << "); }\n";
      }
      f << "  }\n";
      terms_emitted += 2 * static_cast<long long>(row.left.size());
      in_chunk += static_cast<int>(row.left.size());
      if (in_chunk >= 1500) {
        f << "}\n";
        add_fn(sig, f.str());
        post_calls << "  b" << nfunc << "(sv, sa);\n";
        ++nfunc;
        opened = false;
        in_chunk = 0;
      }
    }
    if (opened) {
      f << "}\n";
      add_fn(sig, f.str());
      post_calls << "  b" << nfunc << "(sv, sa);\n";
      ++nfunc;
    }
  }

  // ---- kernel
  std::string all_defs;
  for (const std::string& d : fn_defs) all_defs += d;
  std::ostringstream calls;
  calls << pre_calls.str();
  for (const std::string& fn : energy_fns) calls << "  E += (double)" << fn << "(sv, sa);\n";
  calls << post_calls.str();
  const std::string tag = std::to_string(fnv1a(all_defs + calls.str()) ^ (use_float ? 0x5151ull : 0x1515ull));
  out->kernel_name = "sus2sh_cgsplit_" + tag;
  std::ostringstream src;
  src << "extern \"C\" __global__ void __launch_bounds__(" << block << ", " << min_blocks << ") " << out->kernel_name
      << "(int N, const D4* __restrict__ pos4, const " << T << "* __restrict__ B, " << T
      << "* __restrict__ G, const double* __restrict__ shift, const double* __restrict__ species, "
         "double* __restrict__ pe, int pe_assign) {\n"
      << "  extern __shared__ __align__(16) unsigned char smem_raw[];\n"
      << "  const int i = blockIdx.x * " << block << " + threadIdx.x;\n"
      << "  if (i >= N) return;\n"
      << "  const size_t n = (size_t)N;\n"
      << "  " << T << "* sv = reinterpret_cast<" << T << "*>(smem_raw) + threadIdx.x;\n"
      << "  " << T << "* sa = sv + " << nglob << " * " << block << ";\n";
  src << "  const unsigned long long pol = sus2_pol();\n";
  for (int b = 0; b < Bb; ++b) src << "  " << sv(b) << " = sus2_ld(B + " << basic_canon[b] << " * n + i, pol);\n";
  src << "  for (int s = 0; s < " << nglob << "; ++s) sa[s * " << block << "] = (" << T << ")0;\n"
      << "  double E = 0.0;\n"
      << calls.str()
      << "  const int ti = (int)__double_as_longlong(pos4[i].w);\n"
      << "  const double ct = species[ti];\n"
      << "  const double site = shift[ti] + ct + ct * E;\n"
      << "  if (pe) pe[i] = pe_assign ? site : pe[i] + site;\n"
      << "  const " << T << " sc = (" << T << ")ct;\n";
  std::vector<int> canon_basic(ncanon, -1);
  for (int b = 0; b < Bb; ++b) canon_basic[basic_canon[b]] = b;
  for (int c = 0; c < ncanon; ++c) {
    if (canon_basic[c] >= 0) src << "  sus2_st(G + " << c << " * n + i, sc * " << sa(canon_basic[c]) << ", pol);\n";
    else src << "  sus2_st(G + " << c << " * n + i, (" << T << ")0, pol);\n";
  }
  src << "}\n";
  std::ostringstream head;
  head << "// generated SUS2-SH component-split CG product kernel (" << (use_float ? "FP32" : "FP64") << ", "
       << comps.size() << " components, " << nglob << " shared-memory slots per atom)\n"
       << "struct D4 { double x, y, z, w; };\n" << kCgStreamHelpers;
  // one translation unit, and the same program as parallel units: the kernel
  // with declarations, then the definitions in chunks of similar size
  out->units.clear();
  std::string decls;
  for (const std::string& d : fn_decls) decls += d;
  out->units.push_back(head.str() + decls + src.str());
  const size_t target = std::max<size_t>(all_defs.size() / 32, 200000);
  std::string unit;
  for (const std::string& d : fn_defs) {
    unit += d;
    if (unit.size() >= target) {
      out->units.push_back(unit);
      unit.clear();
    }
  }
  if (!unit.empty()) out->units.push_back(unit);
  if (out->units.size() == 2) out->units.clear();  // one unit of definitions: compile as one program
  out->code = head.str() + all_defs + src.str();
  out->fp_terms = terms_emitted;
  out->block = block;
  out->smem_bytes = 2ull * nglob * block * esz;
  out->functions = nfunc;
  out->components = static_cast<int>(comps.size());
  out->split = true;
  return true;
}

}  // namespace sus2sh
