#include "dftb_params.h"

#include <cstring>
#include <map>
#include <mutex>

#include "dftb_raw.h"
#include "param_files.h"

namespace sgb {

#include "dftb_tables.inc"

namespace {

int n_aos_of(int Z) { return Z <= 2 ? 1 : (Z <= 10 ? 4 : 9); }

std::shared_ptr<const DftbSetData> set_or_null(const char* name) {
  std::string unused;
  return dftb_parameter_set(name, unused);
}

}  // namespace

std::shared_ptr<const DftbSetData> dftb_embedded_set(const std::string& name) {
  static std::mutex mu;
  static std::map<std::string, std::shared_ptr<const DftbSetData>> sets;
  std::lock_guard<std::mutex> lock(mu);
  auto it = sets.find(name);
  if (it != sets.end()) return it->second;
  for (const auto& s : kDftbSetRaw) {
    if (name != s.name) continue;
    auto d = std::make_shared<DftbSetData>();
    d->name = s.name;
    d->elems.assign(kDftbElemRaw + s.elem0, kDftbElemRaw + s.elem0 + s.n_elem);
    for (int i = 0; i < s.n_pair; ++i) {
      DftbPairRaw p = kDftbPairRaw[s.pair0 + i];
      const int row0 = (int)(d->table.size() / 8), spline0 = (int)d->splines.size();
      for (int r = 0; r < p.rows; ++r) d->table.insert(d->table.end(), kDftbTable[p.row0 + r], kDftbTable[p.row0 + r] + 8);
      d->splines.insert(d->splines.end(), kDftbSplineRaw + p.spline0, kDftbSplineRaw + p.spline0 + p.n_spline);
      p.row0 = row0;
      p.spline0 = spline0;
      d->pairs.push_back(p);
    }
    sets[name] = d;
    return d;
  }
  return nullptr;
}

const char* dftb_default_set(Method m) { return m == kDFTB3 ? "3ob-3-1" : "mio-1-1"; }

int dftb_n_aos(const char* set, int Z) {
  auto s = set_or_null(set);
  if (!s || !s->find_elem(Z)) return 0;
  const int n = n_aos_of(Z);
  return n <= 4 ? n : 0;
}

double dftb_core_charge(const char* set, int Z) {
  auto s = set_or_null(set);
  const DftbElemRaw* e = s ? s->find_elem(Z) : nullptr;
  return e ? e->fs + e->fp + e->fd : -1.0;
}

bool dftb_prepare(const std::string& set, int order, const std::vector<int>& Zs, DftbPrepared& out, std::string& err) {
  auto s = dftb_parameter_set(set, err);
  if (!s) return false;
  const int n = (int)Zs.size();
  if (n > kMaxElementSlots) {
    err = "more than 16 distinct elements in one batch";
    return false;
  }
  out.elems.assign(n, DftbElemDev());
  for (int i = 0; i < n; ++i) {
    const DftbElemRaw* e = s->find_elem(Zs[i]);
    if (!e) {
      err = "no " + set + " parameters for element Z=" + std::to_string(Zs[i]);
      return false;
    }
    const int nao = n_aos_of(Zs[i]);
    if (nao > 4) {
      err = "element Z=" + std::to_string(Zs[i]) + " carries d orbitals in DFTB; this engine covers s/p elements only";
      return false;
    }
    if (order == 3 && !e->has_hubbard_derivative) {
      err = "DFTB3 needs a Hubbard derivative for element Z=" + std::to_string(Zs[i]) + " (set " + set + ")";
      return false;
    }
    DftbElemDev& d = out.elems[i];
    d.Z = Zs[i];
    d.nao = nao;
    d.es = e->es;
    d.ep = e->ep;
    d.U = e->us;
    d.occ = e->fs + e->fp + e->fd;
    d.hd = e->hubbard_derivative;
    d.w = nao == 1 ? e->wss : e->wpp;  // SKAtom.h:94-102
    d.has_w = e->has_spin;
    d.pad = 0;
    d.wss = e->wss;
    d.wsp = e->wsp;
    d.wps = e->wps;
    d.wpp = e->wpp;
  }
  out.pairs.assign(kMaxElementSlots * kMaxElementSlots, DftbPairDev());
  out.table.clear();
  out.splines.clear();
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      const DftbPairRaw* r = s->find_pair(Zs[i], Zs[j]);
      const DftbPairRaw* v = s->find_pair(Zs[j], Zs[i]);
      if (!r || !v) {
        err = "no " + set + " Slater-Koster file for the element pair Z=" + std::to_string(Zs[i]) + ", Z=" +
              std::to_string(Zs[j]);
        return false;
      }
      DftbPairDev& p = out.pairs[i * kMaxElementSlots + j];
      p.present = 1;
      p.rows = r->rows;
      p.grid = r->grid;
      p.rmax = r->grid * r->rows + kDftbDistFudge;
      const int na = out.elems[i].nao, nb = out.elems[j].nao;
      p.nint = na + nb == 2 ? 2 : (na + nb == 5 ? 4 : 10);
      // completed table: the eight stored columns, then the reverse pair's
      // s-p overlap and Hamiltonian integrals with opposite sign
      p.table_off = (long long)out.table.size();
      for (int row = 0; row < r->rows; ++row) {
        const double* a = s->table.data() + (size_t)(r->row0 + row) * 8;
        const double* b = row < v->rows ? s->table.data() + (size_t)(v->row0 + row) * 8 : nullptr;
        for (int c = 0; c < 8; ++c) out.table.push_back(a[c]);
        out.table.push_back(b ? -b[2] : 0.0);
        out.table.push_back(b ? -b[3] : 0.0);
      }
      // tail coefficients from the interpolant at the last row (SKPair::precompute5Extrapolation)
      {
        const double* tab = out.table.data() + p.table_off;
        const int start = p.rows - kDftbInter;
        double v1[kDftbCols], d1[kDftbCols], v2[kDftbCols], d2[kDftbCols];
        dftb_interpolate(tab, p.nint, p.grid, (double)(p.rows - 1) - kDftbDeltaR, start, v1, d1);
        dftb_interpolate(tab, p.nint, p.grid, (double)(p.rows - 1) + kDftbDeltaR, start, v2, d2);
        for (int L = 0; L < p.nint; ++L) {
          const double y0 = tab[(size_t)(p.rows - 1) * kDftbCols + L];
          const double y1 = d1[L];
          const double y2 = (d2[L] - d1[L]) / kDftbDeltaR;
          const double x1 = -y1 * (kDftbDistFudge / p.grid);
          const double x2 = y2 * (kDftbDistFudge / p.grid) * (kDftbDistFudge / p.grid);
          p.t3[L] = 10 * y0 - 4 * x1 + 0.5 * x2;
          p.t4[L] = -15 * y0 + 7 * x1 - x2;
          p.t5[L] = 6 * y0 - 3 * x1 + 0.5 * x2;
        }
      }
      // gamma terms of unlike elements (SKPair::precalculateGammaTerms)
      if (Zs[i] != Zs[j]) {
        const double ta = out.elems[i].U * 3.2, tb = out.elems[j].U * 3.2, ta2 = ta * ta, tb2 = tb * tb;
        const double d = ta2 - tb2, e = tb2 - ta2;
        p.g1a = (tb2 * tb2 * ta) / (2.0 * d * d);
        p.g1b = (ta2 * ta2 * tb) / (2.0 * e * e);
        p.g2a = tb2 * tb2 * (tb2 - 3 * ta2) / (d * d * d);
        p.g2b = ta2 * ta2 * (ta2 - 3 * tb2) / (e * e * e);
        p.dgab1a = (tb2 * tb2 * tb2 + 3.0 * ta2 * tb2 * tb2) / (2.0 * d * d * d);
        p.dgab2a = (12.0 * ta2 * ta * tb2 * tb2) / (d * d * d * d);
        p.dgab1b = (2.0 * ta2 * ta * tb2 * tb) / (d * d * d);
        p.dgab2b = (12.0 * ta2 * ta2 * tb2 * tb) / (d * d * d * d);
        p.dgba1a = (ta2 * ta2 * ta2 + 3.0 * tb2 * ta2 * ta2) / (2.0 * e * e * e);
        p.dgba2a = (12.0 * tb2 * tb * ta2 * ta2) / (e * e * e * e);
        p.dgba1b = (2.0 * tb2 * tb * ta2 * ta) / (e * e * e);
        p.dgba2b = (12.0 * tb2 * tb2 * ta2 * ta) / (e * e * e * e);
      }
      // repulsion spline of the file Zi-Zj
      p.n_spline = r->n_spline;
      p.cutoff = r->cutoff;
      p.a1 = r->a1;
      p.a2 = r->a2;
      p.a3 = r->a3;
      p.c4 = r->c4;
      p.c5 = r->c5;
      p.spline_off = (int)out.splines.size();
      for (int k = 0; k < r->n_spline; ++k) {
        const DftbSplineRaw& q = s->splines[r->spline0 + k];
        out.splines.push_back(DftbSplineDev{q.start, q.end, q.c0, q.c1, q.c2, q.c3});
      }
    }
  return true;
}

}  // namespace sgb
