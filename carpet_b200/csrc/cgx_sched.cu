// cgx_sched.cu -- host-side send/recv region logic (the dh schedules) for
// box hierarchies, emitting box-pair lists for cgx_batch_add_many.
//
// CarpetLib builds these lists with bboxset algebra at regrid time
// (CarpetLib/src/dh.cc: sync 837-894, boundary prolongation 896-977,
// restriction 981-1088, old-to-new 1717-1830).  Here the regions of a level
// are given as component boxes (interior: the component's share of the
// level; exterior: grown by the inter-component ghost zones) and refined
// boxes; the lists are built from box intersections and differences.  All
// boxes are int[9] {lower[3], upper[3], stride[3]}, inclusive bounds.
#include <algorithm>
#include <cstring>
#include <vector>

#include "../../include/cgx.h"
#include "cgx_internal.h"

namespace {

struct B {
  int lo[3], up[3], st[3];
  static B from(const int *p) {
    B b;
    for (int d = 0; d < 3; ++d) {
      b.lo[d] = p[d];
      b.up[d] = p[3 + d];
      b.st[d] = p[6 + d];
    }
    return b;
  }
  void to(int *p) const {
    for (int d = 0; d < 3; ++d) {
      p[d] = lo[d];
      p[3 + d] = up[d];
      p[6 + d] = st[d];
    }
  }
  bool empty() const {
    for (int d = 0; d < 3; ++d)
      if (lo[d] > up[d]) return true;
    return false;
  }
  long long npoints() const {
    if (empty()) return 0;
    long long n = 1;
    for (int d = 0; d < 3; ++d) n *= (up[d] - lo[d]) / st[d] + 1;
    return n;
  }
};

B isect(const B &a, const B &b) {
  B c = a;
  for (int d = 0; d < 3; ++d) {
    c.lo[d] = std::max(a.lo[d], b.lo[d]);
    c.up[d] = std::min(a.up[d], b.up[d]);
  }
  return c;
}

// bbox::expand by multiples of the stride (CarpetLib/src/bbox.cc:180-191)
B grow(const B &b, int lo, int up) {
  B c = b;
  for (int d = 0; d < 3; ++d) {
    c.lo[d] -= lo * b.st[d];
    c.up[d] += up * b.st[d];
  }
  return c;
}

// a minus b as disjoint boxes (z slabs, then y, then x)
void subtract(const B &a, const B &b, std::vector<B> &out) {
  const B c = isect(a, b);
  if (c.empty()) {
    if (!a.empty()) out.push_back(a);
    return;
  }
  B rest = a;
  for (int d = 2; d >= 0; --d) {
    if (rest.lo[d] < c.lo[d]) {
      B p = rest;
      p.up[d] = c.lo[d] - a.st[d];
      out.push_back(p);
    }
    if (rest.up[d] > c.up[d]) {
      B p = rest;
      p.lo[d] = c.up[d] + a.st[d];
      out.push_back(p);
    }
    rest.lo[d] = c.lo[d];
    rest.up[d] = c.up[d];
  }
}

std::vector<B> minus_all(const B &a, const std::vector<B> &cut) {
  std::vector<B> parts{a}, nxt;
  for (const B &c : cut) {
    nxt.clear();
    for (const B &p : parts) subtract(p, c, nxt);
    parts.swap(nxt);
  }
  return parts;
}

int fdiv(int a, int b) { return a >= 0 ? a / b : -((-a + b - 1) / b); }
int cdiv(int a, int b) { return -fdiv(-a, b); }

// the smallest coarse-stride box containing b (bbox::expanded_for)
B coarsen_cover(const B &b, int cs) {
  B c;
  for (int d = 0; d < 3; ++d) {
    c.lo[d] = fdiv(b.lo[d], cs) * cs;
    c.up[d] = cdiv(b.up[d], cs) * cs;
    c.st[d] = cs;
  }
  return c;
}

// the largest coarse-stride box inside b (bbox::contracted_for)
B coarsen_inside(const B &b, int cs) {
  B c;
  for (int d = 0; d < 3; ++d) {
    c.lo[d] = cdiv(b.lo[d], cs) * cs;
    c.up[d] = fdiv(b.up[d], cs) * cs;
    c.st[d] = cs;
  }
  return c;
}

std::vector<B> boxes(int n, const int *p) {
  std::vector<B> v((size_t)std::max(n, 0));
  for (int i = 0; i < n; ++i) v[i] = B::from(p + 9 * i);
  return v;
}

struct Out {
  cgx_pair_box *out;
  int max, n;
  void add(int dc, int sc, const B &dst, const B &src) {
    if (n < max) {
      out[n].dst_comp = dc;
      out[n].src_comp = sc;
      dst.to(out[n].dstbox);
      src.to(out[n].srcbox);
    }
    ++n;
  }
  int finish(int *nout) {
    *nout = n;
    if (n > max)
      return cgx::set_error(CGX_ENOMEM, "schedule: %d pairs, room for %d (call again with more)", n, max);
    return CGX_OK;
  }
};

bool args_ok(const void *a, int n) { return n >= 0 && (n == 0 || a); }

// coarse points owned by a coarse component for a fine level of stride fs:
// the interior extended by one coarse cell minus a fine point upward
B owned(const B &ci, int cs, int fs) {
  B o = ci;
  for (int d = 0; d < 3; ++d) {
    o.up[d] = ci.up[d] + cs - fs;
    o.st[d] = fs;
  }
  return o;
}

} // namespace

extern "C" {

int cgx_sched_sync(int ncomp, const int *interior, const int *exterior, cgx_pair_box *out, int max,
                   int *npairs) {
  if (!args_ok(interior, ncomp) || !args_ok(exterior, ncomp) || !npairs || max < 0 || (max && !out))
    return cgx::set_error(CGX_EINVAL, "sched_sync: bad arguments");
  const std::vector<B> in = boxes(ncomp, interior), ex = boxes(ncomp, exterior);
  Out o{out, max, 0};
  std::vector<B> ghosts;
  for (int c = 0; c < ncomp; ++c) {
    ghosts.clear();
    subtract(ex[c], in[c], ghosts);
    for (const B &g : ghosts)
      for (int c2 = 0; c2 < ncomp; ++c2) {
        if (c2 == c) continue;
        const B r = isect(g, in[c2]);
        if (!r.empty()) o.add(c, c2, r, r);
      }
  }
  return o.finish(npairs);
}

int cgx_sched_prolong(int nbox, const int *fboxes, int nfcomp, const int *finterior, int nccomp,
                      const int *cinterior, const int *cexterior, int ghost, int buffer, int order,
                      cgx_pair_box *out, int max, int *npairs) {
  if (!args_ok(fboxes, nbox) || !args_ok(finterior, nfcomp) || !args_ok(cinterior, nccomp) ||
      !args_ok(cexterior, nccomp) || !npairs || max < 0 || (max && !out) || ghost < 0 || buffer < 0)
    return cgx::set_error(CGX_EINVAL, "sched_prolong: bad arguments");
  const std::vector<B> fb = boxes(nbox, fboxes), fi = boxes(nfcomp, finterior);
  const std::vector<B> ci = boxes(nccomp, cinterior), ce = boxes(nccomp, cexterior);
  const int w = ghost + buffer;
  Out o{out, max, 0};
  std::vector<B> shell;
  for (const B &box : fb) {
    shell.clear();
    subtract(box, grow(box, -w, -w), shell);
    const int fs = box.st[0];
    for (int c = 0; c < nfcomp; ++c)
      for (const B &s : shell) {
        const B piece = isect(s, fi[c]);
        if (piece.empty()) continue;
        for (int c2 = 0; c2 < nccomp; ++c2) {
          const int cs = ci[c2].st[0];
          const B r = isect(piece, owned(ci[c2], cs, fs));
          if (r.empty()) continue;
          const B send = grow(coarsen_cover(r, cs), order / 2, order / 2);
          for (int d = 0; d < 3; ++d)
            if (send.lo[d] < ce[c2].lo[d] || send.up[d] > ce[c2].up[d])
              return cgx::set_error(CGX_EINVAL, "sched_prolong: stencil leaves coarse component %d", c2);
          o.add(c, c2, r, send);
        }
      }
  }
  return o.finish(npairs);
}

int cgx_sched_restrict(int nbox, const int *fboxes, int nfcomp, const int *finterior, int nccomp,
                       const int *cinterior, int ghost, int buffer, cgx_pair_box *out, int max,
                       int *npairs) {
  if (!args_ok(fboxes, nbox) || !args_ok(finterior, nfcomp) || !args_ok(cinterior, nccomp) || !npairs ||
      max < 0 || (max && !out))
    return cgx::set_error(CGX_EINVAL, "sched_restrict: bad arguments");
  const std::vector<B> fb = boxes(nbox, fboxes), fi = boxes(nfcomp, finterior), ci = boxes(nccomp, cinterior);
  const int w = ghost + buffer;
  Out o{out, max, 0};
  for (int c2 = 0; c2 < nccomp; ++c2) {
    const int cs = ci[c2].st[0];
    for (int c = 0; c < nfcomp; ++c)
      for (const B &box : fb) {
        const B region = coarsen_inside(isect(grow(box, -w, -w), fi[c]), cs);
        const B r = isect(region, ci[c2]);
        if (r.empty()) continue;
        B send = r;
        for (int d = 0; d < 3; ++d) send.st[d] = fi[c].st[d];
        o.add(c2, c, r, send);
      }
  }
  return o.finish(npairs);
}

int cgx_sched_old2new(int nnew, const int *new_exterior, int nold, const int *old_interior, int nccomp,
                      const int *cinterior, const int *cexterior, int order, cgx_pair_box *copies,
                      int max_copies, int *ncopies, cgx_pair_box *prols, int max_prols, int *nprols) {
  if (!args_ok(new_exterior, nnew) || !args_ok(old_interior, nold) || !args_ok(cinterior, nccomp) ||
      !args_ok(cexterior, nccomp) || !ncopies || !nprols || max_copies < 0 || max_prols < 0 ||
      (max_copies && !copies) || (max_prols && !prols))
    return cgx::set_error(CGX_EINVAL, "sched_old2new: bad arguments");
  const std::vector<B> ne = boxes(nnew, new_exterior), oi = boxes(nold, old_interior);
  const std::vector<B> ci = boxes(nccomp, cinterior), ce = boxes(nccomp, cexterior);
  Out oc{copies, max_copies, 0}, op{prols, max_prols, 0};
  for (int c = 0; c < nnew; ++c) {
    const int fs = ne[c].st[0];
    for (int c2 = 0; c2 < nold; ++c2) {
      const B r = isect(ne[c], oi[c2]);
      if (!r.empty()) oc.add(c, c2, r, r);
    }
    for (const B &piece : minus_all(ne[c], oi))
      for (int c3 = 0; c3 < nccomp; ++c3) {
        const int cs = ci[c3].st[0];
        const B r = isect(piece, owned(ci[c3], cs, fs));
        if (r.empty()) continue;
        const B send = grow(coarsen_cover(r, cs), order / 2, order / 2);
        for (int d = 0; d < 3; ++d)
          if (send.lo[d] < ce[c3].lo[d] || send.up[d] > ce[c3].up[d])
            return cgx::set_error(CGX_EINVAL, "sched_old2new: stencil leaves coarse component %d", c3);
        op.add(c, c3, r, send);
      }
  }
  int rc = oc.finish(ncopies);
  int rc2 = op.finish(nprols);
  return rc ? rc : rc2;
}

} // extern "C"
