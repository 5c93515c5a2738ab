// Discrete normals of boundary cells: the classification boundary::set applies to every cell of
// a boundary material before it picks dynamics and post-processor (computeBoundaryTypeAndNormal,
// geometry/discreteNormals.hh:31-172 in 2D, 176-1191 in 3D).  Host code only.
//
// The reference writes the classification as a cascade of nested conditions on the fluid /
// outside state of the 8 (2D) or 26 (3D) neighbours.  It is restated here as a rule table that a
// small interpreter walks: each rule is a group condition, a rule condition and the result
// (normal type and outward normal).  The order of the rules and the way a later match interacts
// with an earlier one are part of the algorithm and are kept: in 3D the first matching rule of
// the flat, corner and external-edge groups wins and the internal-edge rules overwrite any earlier
// result; in 2D every match overwrites the previous one.  A condition is a list of terms
// "<state><dx><dy>[<dz>]": state F (fluid), N (not fluid), B (neither fluid nor outside) or M
// (outside or not fluid) of the neighbour at the given offset, each offset a sign character '+',
// '-' or '0'.
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/lbx.h"

namespace lbx {
int set_error(int code, const std::string& msg);

namespace {

struct Rule {
  const char* group;  // group condition (the outer if of the reference)
  const char* cond;   // this rule's own condition
  int type;
  int n[3];
  bool overwrite;     // 3D internal edges and every 2D rule replace an earlier match
};

// 3D, in the order of the reference (boundary0N/0P, 1N/1P, 2N/2P, the external corners, the
// internal corners, the external edges, the internal edges).
const Rule kRules3D[] = {
    {"B00+ B00- B0+0 B0-0", "F+00", LBX_NORMAL_FLAT, {-1, 0, 0}, false},
    {"B00+ B00- B0+0 B0-0", "F-00", LBX_NORMAL_FLAT, {1, 0, 0}, false},
    {"B00+ B00- B+00 B-00", "F0+0", LBX_NORMAL_FLAT, {0, -1, 0}, false},
    {"B00+ B00- B+00 B-00", "F0-0", LBX_NORMAL_FLAT, {0, 1, 0}, false},
    {"B+00 B-00 B0+0 B0-0", "F00+", LBX_NORMAL_FLAT, {0, 0, -1}, false},
    {"B+00 B-00 B0+0 B0-0", "F00-", LBX_NORMAL_FLAT, {0, 0, 1}, false},
    {"B+00 B00+ B+0+", "B0+0 B++0 B0++ F+++", LBX_NORMAL_EXTERNAL_CORNER, {-1, -1, -1}, false},
    {"B+00 B00+ B+0+", "B0-0 B+-0 B0-+ F+-+", LBX_NORMAL_EXTERNAL_CORNER, {-1, 1, -1}, false},
    {"B+00 B00- B+0-", "B0-0 B+-0 B0-- F+--", LBX_NORMAL_EXTERNAL_CORNER, {-1, 1, 1}, false},
    {"B+00 B00- B+0-", "B0+0 B++0 B0+- F++-", LBX_NORMAL_EXTERNAL_CORNER, {-1, -1, 1}, false},
    {"B-00 B00- B-0-", "B0-0 B0-- B--0 F---", LBX_NORMAL_EXTERNAL_CORNER, {1, 1, 1}, false},
    {"B-00 B00- B-0-", "B0+0 B0+- B-+0 F-+-", LBX_NORMAL_EXTERNAL_CORNER, {1, -1, 1}, false},
    {"B-00 B00+ B-0+", "B0+0 B0++ B-+0 F-++", LBX_NORMAL_EXTERNAL_CORNER, {1, -1, -1}, false},
    {"B-00 B00+ B-0+", "B0-0 B0-+ B--0 F--+", LBX_NORMAL_EXTERNAL_CORNER, {1, 1, -1}, false},
    {"F-00 F00- B00+ B+00", "F0-0 B0+0", LBX_NORMAL_INTERNAL_CORNER, {1, 1, 1}, false},
    {"F-00 F00- B00+ B+00", "F0+0 B0-0", LBX_NORMAL_INTERNAL_CORNER, {1, -1, 1}, false},
    {"F-00 F00+ B00- B+00", "F0+0 B0-0", LBX_NORMAL_INTERNAL_CORNER, {1, -1, -1}, false},
    {"F-00 F00+ B00- B+00", "F0-0 B0+0", LBX_NORMAL_INTERNAL_CORNER, {1, 1, -1}, false},
    {"F+00 F00- B-00 B00+", "F0-0 B0+0", LBX_NORMAL_INTERNAL_CORNER, {-1, 1, 1}, false},
    {"F+00 F00- B-00 B00+", "F0+0 B0-0", LBX_NORMAL_INTERNAL_CORNER, {-1, -1, 1}, false},
    {"F+00 F00+ B-00 B00-", "F0-0 B0+0", LBX_NORMAL_INTERNAL_CORNER, {-1, 1, -1}, false},
    {"F+00 F00+ B-00 B00-", "F0+0 B0-0", LBX_NORMAL_INTERNAL_CORNER, {-1, -1, -1}, false},
    {"B-00 B+00 B00+ N+0+ N-0+", "F0-+ B0-0", LBX_NORMAL_EXTERNAL_EDGE, {0, 1, -1}, false},
    {"B-00 B+00 B00+ N+0+ N-0+", "F0++ B0+0", LBX_NORMAL_EXTERNAL_EDGE, {0, -1, -1}, false},
    {"B-00 B+00 B00- N+0- N-0-", "F0+- N0+0", LBX_NORMAL_EXTERNAL_EDGE, {0, -1, 1}, false},
    {"B-00 B+00 B00- N+0- N-0-", "F0-- N0-0", LBX_NORMAL_EXTERNAL_EDGE, {0, 1, 1}, false},
    {"B0+0 B0-0 B00+", "F+0+ B+00 N-00 N00-", LBX_NORMAL_EXTERNAL_EDGE, {-1, 0, -1}, false},
    {"B0+0 B0-0 B00+", "F-0+ B-00 N+00 N00-", LBX_NORMAL_EXTERNAL_EDGE, {1, 0, -1}, false},
    {"B0+0 B0-0 B00-", "F+0- B+00 N-00 N00+", LBX_NORMAL_EXTERNAL_EDGE, {-1, 0, 1}, false},
    {"B0+0 B0-0 B00-", "F-0- B-00 N+00 N00+", LBX_NORMAL_EXTERNAL_EDGE, {1, 0, 1}, false},
    {"B00+ B00- B0+0", "N+00 F++0", LBX_NORMAL_EXTERNAL_EDGE, {-1, -1, 0}, false},
    {"B00+ B00- B0+0", "N-00 F-+0", LBX_NORMAL_EXTERNAL_EDGE, {1, -1, 0}, false},
    {"B00+ B00- B0-0", "N-00 F--0", LBX_NORMAL_EXTERNAL_EDGE, {1, 1, 0}, false},
    {"B00+ B00- B0-0", "N+00 F+-0", LBX_NORMAL_EXTERNAL_EDGE, {-1, 1, 0}, false},
    {"B-00 B+00 B00- F00+", "F0+0 B0-0 B--0 B+-0", LBX_NORMAL_INTERNAL_EDGE, {0, -1, -1}, true},
    {"B-00 B+00 B00- F00+", "F0-0 B0+0 B-+0 B++0", LBX_NORMAL_INTERNAL_EDGE, {0, 1, -1}, true},
    {"B+00 B-00 B00+ F00-", "F0+0 B--0 B0-0 B+-0", LBX_NORMAL_INTERNAL_EDGE, {0, -1, 1}, true},
    {"B+00 B-00 B00+ F00-", "F0-0 B-+0 B0+0 B++0", LBX_NORMAL_INTERNAL_EDGE, {0, 1, 1}, true},
    {"F-00 B+00 B0+0 B0-0", "F00- B00+ B0++ B0-+", LBX_NORMAL_INTERNAL_EDGE, {1, 0, 1}, true},
    {"F-00 B+00 B0+0 B0-0", "F00+ B00- B0+- B0--", LBX_NORMAL_INTERNAL_EDGE, {1, 0, -1}, true},
    {"F+00 B-00 B0-0 B0+0", "F00- B00+ B0++ B0-+", LBX_NORMAL_INTERNAL_EDGE, {-1, 0, 1}, true},
    {"F+00 B-00 B0-0 B0+0", "F00+ B00- B0+- B0--", LBX_NORMAL_INTERNAL_EDGE, {-1, 0, -1}, true},
    {"F0-0 B00- B00+ B0+0", "F-00 F--0", LBX_NORMAL_INTERNAL_EDGE, {1, 1, 0}, true},
    {"F0-0 B00- B00+ B0+0", "F+00 F+-0", LBX_NORMAL_INTERNAL_EDGE, {-1, 1, 0}, true},
    {"F0+0 B00- B00+ B0-0", "F-00 F-+0", LBX_NORMAL_INTERNAL_EDGE, {1, -1, 0}, true},
    {"F0+0 B00- B00+ B0-0", "F+00 F++0", LBX_NORMAL_INTERNAL_EDGE, {-1, -1, 0}, true},
};

// 2D (boundary0N/0P, 1N/1P, the external corners, the internal corners); every match overwrites.
const Rule kRules2D[] = {
    {"B0+ B0-", "F+0", LBX_NORMAL_FLAT, {-1, 0, 0}, true},
    {"B0+ B0-", "F-0", LBX_NORMAL_FLAT, {1, 0, 0}, true},
    {"B+0 B-0", "F0+", LBX_NORMAL_FLAT, {0, -1, 0}, true},
    {"B+0 B-0", "F0-", LBX_NORMAL_FLAT, {0, 1, 0}, true},
    {"B+0", "B0+ F++", LBX_NORMAL_EXTERNAL_CORNER, {-1, -1, 0}, true},
    {"B+0", "B0- F+-", LBX_NORMAL_EXTERNAL_CORNER, {-1, 1, 0}, true},
    {"B-0", "B0+ F-+", LBX_NORMAL_EXTERNAL_CORNER, {1, -1, 0}, true},
    {"B-0", "B0- F--", LBX_NORMAL_EXTERNAL_CORNER, {1, 1, 0}, true},
    {"B-0", "B0- M-- F++", LBX_NORMAL_INTERNAL_CORNER, {-1, -1, 0}, true},
    {"B-0", "B0+ M-+ F+-", LBX_NORMAL_INTERNAL_CORNER, {-1, 1, 0}, true},
    {"B+0", "B0- M+- F-+", LBX_NORMAL_INTERNAL_CORNER, {1, -1, 0}, true},
    {"B+0", "B0+ M++ F--", LBX_NORMAL_INTERNAL_CORNER, {1, 1, 0}, true},
};

struct Term {
  char state;
  int off[3];
};

std::vector<Term> parse(const char* s, int d) {
  std::vector<Term> out;
  const char* p = s;
  while (*p) {
    while (*p == ' ') ++p;
    if (!*p) break;
    Term t{*p++, {0, 0, 0}};
    for (int a = 0; a < d; ++a, ++p) t.off[a] = *p == '+' ? 1 : (*p == '-' ? -1 : 0);
    out.push_back(t);
  }
  return out;
}

struct Classifier {
  int d;
  int64_t ext[3];
  int per[3];
  const int32_t* material;
  std::vector<int32_t> fluid, outside;
  struct Parsed {
    std::vector<Term> group, cond;
    const Rule* rule;
  };
  std::vector<Parsed> rules;

  Classifier(int d_, const int32_t core[3], const int32_t periodic[3], const int32_t* mat) : d(d_), material(mat) {
    for (int a = 0; a < 3; ++a) {
      ext[a] = (a < d) ? core[a] : 1;
      per[a] = (periodic && a < d) ? (periodic[a] != 0) : 0;
    }
    const Rule* table = d == 3 ? kRules3D : kRules2D;
    const size_t count = d == 3 ? sizeof(kRules3D) / sizeof(Rule) : sizeof(kRules2D) / sizeof(Rule);
    for (size_t i = 0; i < count; ++i) rules.push_back({parse(table[i].group, d), parse(table[i].cond, d), &table[i]});
  }
  // material of the cell at p (beyond a non-periodic face: 0, the reference's empty overlap)
  int32_t mat(int64_t x, int64_t y, int64_t z) const {
    int64_t p[3] = {x, y, z};
    for (int a = 0; a < 3; ++a) {
      if (p[a] >= 0 && p[a] < ext[a]) continue;
      if (!per[a]) return 0;
      p[a] = ((p[a] % ext[a]) + ext[a]) % ext[a];
    }
    return material[(p[0] * ext[1] + p[1]) * ext[2] + p[2]];
  }
  static bool in(const std::vector<int32_t>& set, int32_t m) {
    for (int32_t v : set)
      if (v == m) return true;
    return false;
  }
  bool holds(const std::vector<Term>& terms, int64_t x, int64_t y, int64_t z) const {
    for (const Term& t : terms) {
      const int32_t m = mat(x + t.off[0], y + t.off[1], z + t.off[2]);
      const bool f = in(fluid, m), o = in(outside, m);
      bool ok;
      switch (t.state) {
      case 'F': ok = f; break;
      case 'N': ok = !f; break;
      case 'M': ok = o || !f; break;
      default: ok = !f && !o;  // 'B'
      }
      if (!ok) return false;
    }
    return true;
  }
  // type and normal of the cell at (x, y, z); false if it is fluid or outside itself
  bool classify(int64_t x, int64_t y, int64_t z, int& type, int n[3]) const {
    const int32_t self = mat(x, y, z);
    if (in(fluid, self) || in(outside, self)) return false;
    type = LBX_NORMAL_FLAT;
    n[0] = n[1] = n[2] = 0;
    bool set = false;
    for (const Parsed& r : rules) {
      if (!holds(r.group, x, y, z) || !holds(r.cond, x, y, z)) continue;
      if (r.rule->overwrite || !set) {
        type = r.rule->type;
        for (int a = 0; a < 3; ++a) n[a] = r.rule->n[a];
        set = true;
      }
    }
    return true;
  }
};

}  // namespace

// Classifies every core cell of material `boundary`; see lbx_discrete_normals.
int discrete_normals(int q, const int32_t core[3], const int32_t periodic[3], const int32_t* material,
                     int32_t boundary, int32_t n_fluid, const int32_t* fluid, int32_t n_outside,
                     const int32_t* outside, std::vector<int64_t>& cells, std::vector<int32_t>& types,
                     std::vector<int32_t>& normals) {
  if (!core || !material || (n_fluid > 0 && !fluid) || (n_outside > 0 && !outside) || n_fluid < 0 || n_outside < 0)
    return set_error(LBX_ERR_INVALID, "null or negative argument");
  if (q != 9 && q != 19 && q != 27) return set_error(LBX_ERR_UNSUPPORTED, "descriptor must be D2Q9, D3Q19 or D3Q27");
  const int d = q == 9 ? 2 : 3;
  if (core[0] < 1 || core[1] < 1 || (d == 3 && core[2] < 1)) return set_error(LBX_ERR_INVALID, "core extents must be >= 1");
  Classifier cl(d, core, periodic, material);
  cl.fluid.assign(fluid, fluid + n_fluid);
  cl.outside.assign(outside, outside + n_outside);
  cells.clear();
  types.clear();
  normals.clear();
  const int64_t nz = d == 3 ? core[2] : 1;
  for (int64_t x = 0; x < core[0]; ++x)
    for (int64_t y = 0; y < core[1]; ++y)
      for (int64_t z = 0; z < nz; ++z) {
        const int64_t c = (x * core[1] + y) * nz + z;
        if (material[c] != boundary) continue;
        int type = 0, n[3] = {0, 0, 0};
        if (!cl.classify(x, y, z, type, n)) {
          type = -1;  // the boundary material is also a fluid or outside material
        }
        cells.push_back(c);
        types.push_back(type);
        for (int a = 0; a < 3; ++a) normals.push_back(n[a]);
      }
  return LBX_OK;
}

}  // namespace lbx

extern "C" int lbx_discrete_normals(int32_t q, const int32_t core[3], const int32_t periodic[3],
                                    const int32_t* material, int32_t boundary, int32_t n_fluid, const int32_t* fluid,
                                    int32_t n_outside, const int32_t* outside, int64_t cap, int64_t* cells,
                                    int32_t* types, int32_t* normals, int64_t* n_out) {
  if (!n_out || cap < 0) return lbx::set_error(LBX_ERR_INVALID, "null n_out or negative capacity");
  std::vector<int64_t> c;
  std::vector<int32_t> t, n;
  const int rc = lbx::discrete_normals(q, core, periodic, material, boundary, n_fluid, fluid, n_outside, outside, c, t, n);
  if (rc != LBX_OK) return rc;
  *n_out = int64_t(c.size());
  for (int64_t k = 0; k < int64_t(c.size()) && k < cap; ++k) {
    if (cells) cells[k] = c[size_t(k)];
    if (types) types[k] = t[size_t(k)];
    if (normals)
      for (int a = 0; a < 3; ++a) normals[3 * k + a] = n[size_t(3 * k + a)];
  }
  return LBX_OK;
}
