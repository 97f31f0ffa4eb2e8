// cgx_dh.cu -- the dh schedule producer for arbitrary component sets (host).
//
// The region algebra of CarpetLib's dh::regrid (CarpetLib/src/dh.cc:300-1088)
// for vertex-centred hierarchies with refinement factor 2: from every
// level's domain and component interiors it derives each component's
// exterior, ghost zones, communicated and owned regions, buffer zones and
// active region (dh.cc:300-600), and from those the three send/recv lists
// of the transfer path:
//
//   sync     ghost zones from the other components' interiors, components
//            in order (dh.cc:837-894);
//   bndprol  what sync cannot fill, the buffer zones, from the coarser
//            level's components whose active region (expanded by one
//            coarse point) covers the point, the send box being the
//            receive box's coarse cover grown by the stencil size
//            order / 2 (dh.cc:896-977);
//   restrict the coarse points under the fine active region, into every
//            coarse component's exterior (CarpetLib restricts into ghost
//            zones unless higher-order restriction is on) or interior only,
//            from the fine components in order (dh.cc:981-1088).
//
// Sets of points are kept as lists of disjoint boxes of one stride (the
// role of bboxset); the decomposition into boxes is this file's own, so the
// lists' boxes may be cut differently from CarpetLib's, while every point is
// received once, from the same component the reference's order picks.  The
// checks of the reference (every point received, send boxes inside the
// source exterior) become CGX_EINVAL with the reference's message.
#include <algorithm>
#include <string>
#include <vector>

#include "../../include/cgx.h"
#include "cgx_internal.h"

namespace {

struct B {
  int lo[3], up[3], st[3];
  bool empty() const {
    for (int d = 0; d < 3; ++d)
      if (lo[d] > up[d]) return true;
    return false;
  }
  long long size() const {
    if (empty()) return 0;
    long long n = 1;
    for (int d = 0; d < 3; ++d) n *= (up[d] - lo[d]) / st[d] + 1;
    return n;
  }
};

B from9(const int *p) {
  B b;
  for (int d = 0; d < 3; ++d) {
    b.lo[d] = p[d];
    b.up[d] = p[3 + d];
    b.st[d] = p[6 + d];
  }
  return b;
}
void to9(const B &b, int *p) {
  for (int d = 0; d < 3; ++d) {
    p[d] = b.lo[d];
    p[3 + d] = b.up[d];
    p[6 + d] = b.st[d];
  }
}

int floordiv(int a, int b) { return a >= 0 ? a / b : -((-a + b - 1) / b); }
int imod(int a, int b) { return a - b * floordiv(a, b); }

B isect(const B &a, const B &b) {
  B r = a;
  for (int d = 0; d < 3; ++d) {
    r.lo[d] = std::max(a.lo[d], b.lo[d]);
    r.up[d] = std::min(a.up[d], b.up[d]);
  }
  return r;
}
bool contains(const B &outer, const B &b) {
  if (b.empty()) return true;
  for (int d = 0; d < 3; ++d)
    if (b.lo[d] < outer.lo[d] || b.up[d] > outer.up[d]) return false;
  return true;
}
// bbox::expand by stride units (bbox.cc:180-191)
B expand(const B &b, const int lo[3], const int up[3]) {
  B r = b;
  for (int d = 0; d < 3; ++d) {
    r.lo[d] -= lo[d] * b.st[d];
    r.up[d] += up[d] * b.st[d];
  }
  return r;
}
B expand_all(const B &b, int n) {
  const int v[3] = {n, n, n};
  return expand(b, v, v);
}
// bbox::expanded_for (bbox.cc:210-219): the smallest box on the lattice of
// l (its stride and offset) containing b
B expanded_for(const B &b, const B &l) {
  B r;
  for (int d = 0; d < 3; ++d) {
    const int s = l.st[d];
    r.st[d] = s;
    if (b.empty()) {
      r.lo[d] = l.lo[d];
      r.up[d] = l.lo[d] - s;
      continue;
    }
    r.lo[d] = b.lo[d] - imod(b.lo[d] - l.lo[d], s);
    const int uoff = imod(b.up[d] - l.lo[d], s);
    r.up[d] = b.up[d] + (s - uoff) % s;
  }
  return r;
}
// bbox::contracted_for (bbox.cc:223-232): the largest box on l's lattice
// inside b
B contracted_for(const B &b, const B &l) {
  B r;
  for (int d = 0; d < 3; ++d) {
    const int s = l.st[d];
    r.st[d] = s;
    if (b.empty()) {
      r.lo[d] = l.lo[d];
      r.up[d] = l.lo[d] - s;
      continue;
    }
    const int loff = imod(b.lo[d] - l.lo[d], s);
    r.lo[d] = b.lo[d] + (s - loff) % s;
    r.up[d] = b.up[d] - imod(b.up[d] - l.lo[d], s);
  }
  return r;
}

// a minus b as disjoint boxes (slabs in z, then y, then x)
void minus_into(const B &a, const B &b, std::vector<B> &out) {
  const B c = isect(a, b);
  if (c.empty()) {
    if (!a.empty()) out.push_back(a);
    return;
  }
  B rest = a;
  for (int d = 2; d >= 0; --d) {
    if (rest.lo[d] < c.lo[d]) {
      B s = rest;
      s.up[d] = c.lo[d] - a.st[d];
      out.push_back(s);
    }
    if (rest.up[d] > c.up[d]) {
      B s = rest;
      s.lo[d] = c.up[d] + a.st[d];
      out.push_back(s);
    }
    rest.lo[d] = c.lo[d];
    rest.up[d] = c.up[d];
  }
}

// a set of points of one stride as disjoint boxes (the role of bboxset)
struct BSet {
  std::vector<B> v;
  bool empty() const { return v.empty(); }
  BSet minus(const B &b) const {
    BSet r;
    for (const B &a : v) minus_into(a, b, r.v);
    return r;
  }
  BSet minus(const BSet &s) const {
    BSet r = *this;
    for (const B &b : s.v) r = r.minus(b);
    return r;
  }
  BSet isect(const B &b) const {
    BSet r;
    for (const B &a : v) {
      const B c = ::isect(a, b);
      if (!c.empty()) r.v.push_back(c);
    }
    return r;
  }
  BSet isect(const BSet &s) const {
    BSet r;
    for (const B &b : s.v) {
      const BSet p = isect(b);
      r.v.insert(r.v.end(), p.v.begin(), p.v.end());
    }
    return r;
  }
  void add(const B &b) { // union
    if (b.empty()) return;
    BSet p;
    p.v.push_back(b);
    p = p.minus(*this);
    v.insert(v.end(), p.v.begin(), p.v.end());
  }
  void add(const BSet &s) {
    for (const B &b : s.v) add(b);
  }
  // bboxset::expand: every box grown by n stride units, united
  BSet expanded(int n) const {
    BSet r;
    for (const B &b : v) r.add(expand_all(b, n));
    return r;
  }
  BSet expanded_for(const B &l) const {
    BSet r;
    for (const B &b : v) r.add(::expanded_for(b, l));
    return r;
  }
  BSet contracted_for(const B &l) const {
    BSet r;
    for (const B &b : v) r.add(::contracted_for(b, l));
    return r;
  }
  // merge boxes that continue each other along one axis with equal
  // extents in the other two, until none do (as bboxset normalises): the
  // same points in fewer, larger boxes
  BSet normalized() const {
    std::vector<B> w = v;
    for (bool changed = true; changed;) {
      changed = false;
      for (int d = 0; d < 3; ++d)
        for (size_t i = 0; i < w.size(); ++i)
          for (size_t j = i + 1; j < w.size();) {
            const B &a = w[i], &b = w[j];
            bool same = true;
            for (int e = 0; e < 3; ++e)
              if (e != d && (a.lo[e] != b.lo[e] || a.up[e] != b.up[e])) same = false;
            if (same && (a.up[d] + a.st[d] == b.lo[d] || b.up[d] + b.st[d] == a.lo[d])) {
              B m = a;
              m.lo[d] = std::min(a.lo[d], b.lo[d]);
              m.up[d] = std::max(a.up[d], b.up[d]);
              w[i] = m;
              w.erase(w.begin() + (long)j);
              changed = true;
            } else {
              ++j;
            }
          }
    }
    BSet r;
    r.v = w;
    return r;
  }
};
BSet single(const B &b) {
  BSet s;
  if (!b.empty()) s.v.push_back(b);
  return s;
}

struct Comp {
  B intr, extr, comm, owned;
  BSet ghosts, buffers, active, sync;
};
struct Level {
  B domain;
  std::vector<Comp> comps;
  BSet allactive;
  std::vector<cgx_pair_box> sync, bndprol, restrict_; // restrict_: into this level from the next finer
};

} // namespace

struct cgx_dh {
  std::vector<Level> levels;
};

namespace {

int err(const char *what, int l, int c) {
  return cgx::set_error(CGX_EINVAL, "dh: %s (level %d, component %d)", what, l, c);
}
void push(std::vector<cgx_pair_box> &out, int dst, int src, const B &recv, const B &send) {
  cgx_pair_box p;
  p.dst_comp = dst;
  p.src_comp = src;
  to9(recv, p.dstbox);
  to9(send, p.srcbox);
  out.push_back(p);
}

// dh.cc:300-600: the component and level regions of one level
int regions(Level &L, int l, int ghost, int buffer, int bw) {
  const B &D = L.domain;
  const B dactive = expand_all(D, -bw);
  BSet allowned;
  for (size_t c = 0; c < L.comps.size(); ++c) {
    Comp &k = L.comps[c];
    if (!contains(D, k.intr)) return err("The interior must be contained in the domain", l, (int)c);
    int gl[3], gu[3], bl[3], bu[3];
    for (int d = 0; d < 3; ++d) {
      const bool ol = k.intr.lo[d] == D.lo[d], ou = k.intr.up[d] == D.up[d];
      gl[d] = ol ? 0 : ghost;
      gu[d] = ou ? 0 : ghost;
      bl[d] = ol ? -bw : 0;
      bu[d] = ou ? -bw : 0;
    }
    k.extr = expand(k.intr, gl, gu);
    if (!contains(D, k.extr)) return err("The exterior must be contained in the domain", l, (int)c);
    k.ghosts = single(k.extr).minus(k.intr);
    k.comm = expand(k.extr, bl, bu);
    k.owned = expand(k.intr, bl, bu);
    for (const Comp &o : L.comps)
      if (&o != &k && !isect(o.intr, k.intr).empty())
        return err("All interiors must be disjunct", l, (int)c);
    allowned.add(k.owned);
  }
  const BSet notowned = single(dactive).minus(allowned);
  const BSet notactive = notowned.expanded(buffer);
  const BSet allbuffers = allowned.isect(notactive);
  L.allactive = allowned.minus(notactive);
  for (Comp &k : L.comps) {
    k.buffers = allbuffers.isect(k.owned);
    k.active = L.allactive.isect(k.owned);
  }
  return CGX_OK;
}

// dh.cc:837-894
int sync_list(Level &L, int l) {
  for (size_t c = 0; c < L.comps.size(); ++c) {
    Comp &k = L.comps[c];
    BSet need = k.ghosts;
    for (size_t cc = 0; cc < L.comps.size() && !need.empty(); ++cc) {
      const BSet ovlp = need.isect(L.comps[cc].intr).normalized();
      if (cc == c && !ovlp.empty()) return err("A region may not synchronise from itself", l, (int)c);
      for (const B &r : ovlp.v) push(L.sync, (int)c, (int)cc, r, r);
      need = need.minus(ovlp);
      k.sync.add(ovlp);
    }
  }
  return CGX_OK;
}

// dh.cc:896-977
int bndprol_list(Level &F, const Level &C, int l, int order) {
  const int stencil = order / 2;
  for (size_t c = 0; c < F.comps.size(); ++c) {
    Comp &k = F.comps[c];
    BSet need = k.ghosts.minus(k.sync).isect(k.comm);
    need.add(k.buffers);
    for (size_t cc = 0; cc < C.comps.size() && !need.empty(); ++cc) {
      const Comp &o = C.comps[cc];
      // vertex centring: the coarse active region on the fine lattice,
      // grown by the refinement factor (2 fine points)
      const BSet eoa = o.active.expanded_for(k.intr).expanded(2);
      const BSet ovlp = need.isect(eoa).normalized();
      for (const B &r : ovlp.v) {
        const B send = expand_all(expanded_for(r, o.intr), stencil);
        if (!contains(o.extr, send))
          return err("Boundary prolongation: Send region must be contained in exterior", l, (int)c);
        push(F.bndprol, (int)c, (int)cc, r, send);
      }
      need = need.minus(ovlp);
    }
    if (!need.empty())
      return err("Synchronisation and boundary prolongation: All points must have been received", l, (int)c);
  }
  return CGX_OK;
}

// dh.cc:981-1088 (vertex centring)
int restrict_list(Level &F, Level &C, int l, bool into_ghosts) {
  const BSet allrestricted = F.allactive.contracted_for(C.domain);
  for (size_t oc = 0; oc < C.comps.size(); ++oc) {
    const Comp &o = C.comps[oc];
    BSet need = allrestricted.isect(into_ghosts ? o.extr : o.intr);
    if (!need.isect(o.buffers).empty()) return err("Cannot restrict into buffer zones", l - 1, (int)oc);
    for (size_t c = 0; c < F.comps.size() && !need.empty(); ++c) {
      const Comp &k = F.comps[c];
      const BSet ce = single(contracted_for(k.extr, C.domain));
      const BSet ovlp = need.isect(ce).normalized();
      for (const B &r : ovlp.v) {
        const B send = expanded_for(r, k.extr);
        if (!contains(k.extr, send))
          return err("Refinement restriction: Send region must be contained in exterior", l, (int)c);
        push(C.restrict_, (int)oc, (int)c, r, send);
      }
      need = need.minus(ovlp);
    }
    if (!need.empty()) return err("Refinement restriction: All points must have been received", l - 1, (int)oc);
  }
  return CGX_OK;
}

} // namespace

extern "C" {

int cgx_dh_create(cgx_dh **out, int nlevels, const int *domains, const int *ncomps, const int *interiors,
                  int ghost, int buffer, int boundary_width, int order, int restrict_into_ghosts) {
  if (!out || nlevels <= 0 || !domains || !ncomps || !interiors || ghost < 0 || buffer < 0 ||
      boundary_width < 0 || order < 0)
    return cgx::set_error(CGX_EINVAL, "dh: bad arguments");
  cgx_dh *h = new cgx_dh();
  h->levels.resize(nlevels);
  const int *ip = interiors;
  for (int l = 0; l < nlevels; ++l) {
    Level &L = h->levels[l];
    L.domain = from9(domains + 9 * l);
    if (ncomps[l] < 0) {
      delete h;
      return cgx::set_error(CGX_EINVAL, "dh: negative component count");
    }
    for (int c = 0; c < ncomps[l]; ++c, ip += 9) {
      Comp k;
      k.intr = from9(ip);
      L.comps.push_back(k);
    }
    for (int d = 0; d < 3; ++d)
      if (l > 0 && L.domain.st[d] * 2 != h->levels[l - 1].domain.st[d]) {
        delete h;
        return cgx::set_error(CGX_EINVAL, "dh: refinement factor 2 between levels %d and %d", l - 1, l);
      }
  }
  int rc = CGX_OK;
  for (int l = 0; l < nlevels && rc == CGX_OK; ++l) rc = regions(h->levels[l], l, ghost, buffer, boundary_width);
  for (int l = 0; l < nlevels && rc == CGX_OK; ++l) {
    rc = sync_list(h->levels[l], l);
    if (rc == CGX_OK && l > 0) rc = bndprol_list(h->levels[l], h->levels[l - 1], l, order);
    if (rc == CGX_OK && l > 0) rc = restrict_list(h->levels[l], h->levels[l - 1], l, restrict_into_ghosts != 0);
  }
  if (rc) {
    delete h;
    return rc;
  }
  *out = h;
  return CGX_OK;
}

int cgx_dh_destroy(cgx_dh *h) {
  delete h;
  return CGX_OK;
}

int cgx_dh_exteriors(const cgx_dh *h, int level, int *out) {
  if (!h || level < 0 || level >= (int)h->levels.size() || !out) return cgx::set_error(CGX_EINVAL, "dh: bad level");
  const Level &L = h->levels[level];
  for (size_t c = 0; c < L.comps.size(); ++c) to9(L.comps[c].extr, out + 9 * c);
  return CGX_OK;
}

int cgx_dh_pairs(const cgx_dh *h, int level, int kind, cgx_pair_box *out, int max, int *n) {
  if (!h || level < 0 || level >= (int)h->levels.size() || !n || max < 0 || (max && !out))
    return cgx::set_error(CGX_EINVAL, "dh: bad arguments");
  const Level &L = h->levels[level];
  const std::vector<cgx_pair_box> *v = kind == CGX_DH_SYNC ? &L.sync
                                       : kind == CGX_DH_BNDPROL ? &L.bndprol
                                       : kind == CGX_DH_RESTRICT ? &L.restrict_
                                                                 : nullptr;
  if (!v) return cgx::set_error(CGX_EINVAL, "dh: unknown schedule %d", kind);
  *n = (int)v->size();
  if ((int)v->size() > max) return cgx::set_error(CGX_EINVAL, "dh: %zu pairs, room for %d", v->size(), max);
  std::copy(v->begin(), v->end(), out);
  return CGX_OK;
}

} // extern "C"
