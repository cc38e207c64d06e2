// Divide-and-conquer SCF of a molecule, restated on the CPU: pm7-rs src/dandc/mod.rs:143-428
// (run_dandc), src/dandc/partition.rs (bisect, grow_buffer, weights) and src/dandc/sparse.rs
// (pattern, rms_diff, mix, population), with the energy of dandc_derivatives (:446-506).
//
// TEST INFRASTRUCTURE ONLY: the correctness oracle of pm7_run_dandc. The product never links or
// calls it. The global density is a dense matrix with zeros outside the stored atom-pair pattern,
// which holds exactly the numbers of the reference's block-sparse store. Buffer atoms are taken
// in ascending index order (the reference takes them in the order of its cell grid); the order
// of a subsystem's atoms changes its sums only by rounding.
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "oracle_internal.hpp"

namespace oracle {
namespace {

struct Part {
  std::vector<int> parent;  // core atoms, then the buffer
  int n_core = 0;
  double weight(int i, int j) const {  // src/dandc/partition.rs Subsystem::weight
    const bool ci = i < n_core, cj = j < n_core;
    return (ci && cj) ? 1.0 : ((ci || cj) ? 0.5 : 0.0);
  }
};

// partition.rs bisect: split at the median of a stable sort along the longest extent (the last
// of equal extents, as Iterator::max_by picks it) until a part has at most `target` atoms.
void bisect(std::vector<int> idx, const Molecule &mol, size_t target, std::vector<std::vector<int>> &out) {
  if (idx.size() <= target || idx.size() < 2) {
    out.push_back(std::move(idx));
    return;
  }
  double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int i : idx)
    for (int k = 0; k < 3; ++k) {
      lo[k] = std::min(lo[k], mol.pos[i].get(k));
      hi[k] = std::max(hi[k], mol.pos[i].get(k));
    }
  int axis = 0;
  for (int k = 1; k < 3; ++k)
    if (hi[k] - lo[k] >= hi[axis] - lo[axis]) axis = k;
  std::stable_sort(idx.begin(), idx.end(),
                   [&](int a, int b) { return mol.pos[a].get(axis) < mol.pos[b].get(axis); });
  const size_t half = idx.size() / 2;
  std::vector<int> right(idx.begin() + (std::ptrdiff_t)half, idx.end());
  idx.resize(half);
  bisect(std::move(idx), mol, target, out);
  bisect(std::move(right), mol, target, out);
}

// partition.rs partition + grow_buffer (molecule): every atom within `buffer` of a core atom.
std::vector<Part> partition(const Molecule &mol, int core_size, double buffer) {
  std::vector<std::vector<int>> cores;
  std::vector<int> all(mol.size());
  for (int i = 0; i < mol.size(); ++i) all[i] = i;
  bisect(std::move(all), mol, (size_t)std::max(core_size, 1), cores);
  std::vector<Part> parts;
  std::vector<char> in_core(mol.size());
  for (auto &c : cores) {
    Part p;
    p.parent = c;
    p.n_core = (int)c.size();
    std::fill(in_core.begin(), in_core.end(), 0);
    for (int i : c) in_core[i] = 1;
    for (int j = 0; j < mol.size(); ++j) {
      if (in_core[j]) continue;
      for (int i : c)
        if ((mol.pos[j] - mol.pos[i]).norm2() <= buffer * buffer) {
          p.parent.push_back(j);
          break;
        }
    }
    parts.push_back(std::move(p));
  }
  return parts;
}

double occupation(double e, double fermi, double width) {  // src/dandc/mod.rs:563-573
  const double x = (e - fermi) / width;
  if (x > 40.0) return 0.0;
  if (x < -40.0) return 2.0;
  return 2.0 / (1.0 + std::exp(x));
}

struct Solution {
  std::vector<double> ea, va, eb, vb;  // eigenvalues, eigenvectors as rows
  Basis basis;
  double energy = 0.0;
};

struct Cluster {
  Molecule mol;
  Basis basis;
  CoreHamiltonian core;
};

void run_dandc(const Molecule &mol, const pm7_options &o, const pm7_dandc_options &dc, pm7_dandc_result *r) {
  validate_input(mol, o);
  auto bad = [](const char *s) { throw Error(PM7_ERR_INVALID_INPUT, s); };  // src/dandc/mod.rs:83-110
  if (!std::isfinite(dc.buffer) || dc.buffer <= 0.0) bad("the divide-and-conquer buffer must be finite and positive");
  if (dc.core_size <= 0) bad("the divide-and-conquer core size must be at least 1");
  if (!std::isfinite(dc.fermi_width_ev) || dc.fermi_width_ev <= 0.0)
    bad("the divide-and-conquer Fermi width must be finite and positive");
  if (!(dc.mixing > 0.0 && dc.mixing <= 1.0)) bad("the divide-and-conquer mixing factor must lie in (0, 1]");
  const Params &p = params_for(o.method);
  const Basis basis = build_basis(mol, p);
  const int N = mol.size(), nao = basis.nao;
  std::vector<Part> parts = partition(mol, dc.core_size, dc.buffer);

  int largest = 0, largest_atoms = 0;
  for (const Part &s : parts) {
    int k = 0;
    for (int a : s.parent) k += basis.atom_norb[a];
    largest = std::max(largest, k);
    largest_atoms = std::max(largest_atoms, (int)s.parent.size());
  }
  bool has_d = o.force_dpath != 0;
  for (int z : mol.z) has_d = has_d || p.element(z).has_d();
  try {
    memory_guard(largest, (size_t)largest_atoms * (size_t)std::max(largest_atoms - 1, 0) / 2, has_d, o.max_memory_mb);
  } catch (const Error &e) {
    throw Error(PM7_ERR_INVALID_INPUT, std::string(e.what()) + "\nThis is a divide-and-conquer subsystem, not the whole system");
  }

  // pattern and realised weight totals (src/dandc/mod.rs:203-258)
  std::vector<double> wtot((size_t)N * N, 0.0);
  for (const Part &s : parts)
    for (int i = 0; i < (int)s.parent.size(); ++i)
      for (int j = 0; j < (int)s.parent.size(); ++j) {
        const double w = s.weight(i, j);
        if (w > 0.0) wtot[(size_t)s.parent[i] * N + s.parent[j]] += w;
      }
  auto stored = [&](int a, int b) { return wtot[(size_t)a * N + b] > 0.0; };
  int64_t n_stored = 0;
  for (int a = 0; a < N; ++a)
    for (int b = 0; b < N; ++b)
      if (stored(a, b)) n_stored += (int64_t)basis.atom_norb[a] * basis.atom_norb[b];

  double core_e = 0.0;
  for (int z : mol.z) core_e += p.element(z).core_charge;
  const double n_elec = core_e - o.charge;
  if (n_elec < -1.0e-9) bad("the divide-and-conquer driver was given a system with negative electron count");
  const bool uhf = o.reference == PM7_REF_UNRESTRICTED || (o.reference == PM7_REF_AUTO && o.multiplicity > 1);
  const double n_beta_extra = (o.multiplicity - 1) * 0.5;

  Mat P(nao), S(nao);
  {
    const Mat guess = sad_density(mol, basis, p, n_elec);  // diagonal blocks (:289-301)
    for (int a = 0; a < N; ++a) {
      const int off = basis.atom_offset[a], na = basis.atom_norb[a];
      for (int i = 0; i < na; ++i)
        for (int j = 0; j < na; ++j) P(off + i, off + j) = guess(off + i, off + j);
    }
    if (uhf) {  // (:302-323)
      const double scale = core_e > 0.0 ? 2.0 * n_beta_extra / core_e : 0.0;
      for (int k = 0; k < nao; ++k) S(k, k) = scale * P(k, k);
    }
  }
  std::vector<double> cores(N);
  for (int a = 0; a < N; ++a) cores[a] = p.element(mol.z[a]).core_charge;
  auto coulomb = [&](const std::vector<double> &q) {  // far_field / FarField::electronic (molecule)
    std::vector<double> out(N, 0.0);
    for (int a = 0; a < N; ++a) {
      double s = 0.0;
      for (int b = 0; b < N; ++b)
        if (b != a) s += EV * q[b] / (mol.pos[b] - mol.pos[a]).norm();
      out[a] = s;
    }
    return out;
  };
  const std::vector<double> gnuc = coulomb(cores);

  // the subsystems' own core Hamiltonians depend on the geometry only
  std::vector<Cluster> clusters(parts.size());
#pragma omp parallel for schedule(dynamic)
  for (size_t s = 0; s < parts.size(); ++s) {
    Cluster &c = clusters[s];
    for (int a : parts[s].parent) {
      c.mol.z.push_back(mol.z[a]);
      c.mol.pos.push_back(mol.pos[a]);
    }
    c.basis = build_basis(c.mol, p);
    c.core = build_core(c.mol, c.basis, p, false);  // hamiltonian::build_core(&cluster, ...)
  }

  auto pops_of = [&](const Mat &D) {  // SparseDensity::population
    std::vector<double> pop(N, 0.0);
    for (int a = 0; a < N; ++a)
      for (int m = 0; m < basis.atom_norb[a]; ++m) pop[a] += D(basis.atom_offset[a] + m, basis.atom_offset[a] + m);
    return pop;
  };

  double fermi = 0.0, err = INFINITY, electronic = 0.0;
  int iterations = 0;
  bool converged = false;
  std::vector<Solution> sol(parts.size());
  for (int iter = 0; iter < dc.max_scf; ++iter) {
    iterations = iter + 1;
    const std::vector<double> pops = pops_of(P);
    const std::vector<double> gelec = coulomb(pops);
    // solve_subsystem (src/dandc/mod.rs:526-663)
#pragma omp parallel for schedule(dynamic)
    for (size_t s = 0; s < parts.size(); ++s) {
      const Part &pt = parts[s];
      const Cluster &c = clusters[s];
      const int n = (int)pt.parent.size(), m = c.basis.nao;
      std::vector<double> vn(n), ve(n);
      for (int i = 0; i < n; ++i) {  // environment_field (:946-998)
        double zs = 0.0, ps = 0.0;
        for (int j = 0; j < n; ++j) {
          if (i == j) continue;
          const double rr = (c.mol.pos[j] - c.mol.pos[i]).norm();
          if (rr < 1.0e-8) continue;
          zs += EV * cores[pt.parent[j]] / rr;
          ps += EV * pops[pt.parent[j]] / rr;
        }
        vn[i] = gnuc[pt.parent[i]] - zs;
        ve[i] = gelec[pt.parent[i]] - ps;
      }
      CoreHamiltonian core = c.core;
      for (int i = 0; i < n; ++i)
        for (int mu = 0; mu < c.basis.atom_norb[i]; ++mu) core.h(c.basis.atom_offset[i] + mu, c.basis.atom_offset[i] + mu) -= vn[i];
      auto local = [&](const Mat &G) {  // local_density (:672-690)
        Mat L(m);
        for (int i = 0; i < n; ++i)
          for (int j = 0; j < n; ++j) {
            if (!stored(pt.parent[i], pt.parent[j])) continue;
            const int gi = basis.atom_offset[pt.parent[i]], gj = basis.atom_offset[pt.parent[j]];
            const int li = c.basis.atom_offset[i], lj = c.basis.atom_offset[j];
            for (int mu = 0; mu < c.basis.atom_norb[i]; ++mu)
              for (int nu = 0; nu < c.basis.atom_norb[j]; ++nu) L(li + mu, lj + nu) = G(gi + mu, gj + nu);
          }
        return L;
      };
      const Mat pl = local(P);
      auto add_env = [&](Mat &f) {
        for (int i = 0; i < n; ++i)
          for (int mu = 0; mu < c.basis.atom_norb[i]; ++mu) f(c.basis.atom_offset[i] + mu, c.basis.atom_offset[i] + mu) += ve[i];
      };
      Mat fa, fb;
      if (!uhf) {
        Mat half(m);
        for (size_t k = 0; k < half.a.size(); ++k) half.a[k] = 0.5 * pl.a[k];
        fa = build_fock_spin(c.mol, c.basis, p, core, pl, half);
      } else {
        const Mat sl = local(S);
        Mat pa(m), pb(m);
        for (size_t k = 0; k < pa.a.size(); ++k) {
          pa.a[k] = 0.5 * (pl.a[k] + sl.a[k]);
          pb.a[k] = 0.5 * (pl.a[k] - sl.a[k]);
        }
        fa = build_fock_spin(c.mol, c.basis, p, core, pl, pa);
        fb = build_fock_spin(c.mol, c.basis, p, core, pl, pb);
        add_env(fb);
      }
      add_env(fa);
      Solution &so = sol[s];
      so.basis = c.basis;
      symmetric_eigen(fa, so.ea, so.va);
      if (uhf) symmetric_eigen(fb, so.eb, so.vb);
      double e = 0.0;  // (:634-653), with the alpha Fock
      for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
          const double w = pt.weight(i, j);
          if (w == 0.0) continue;
          const int oi = c.basis.atom_offset[i], oj = c.basis.atom_offset[j];
          for (int mu = 0; mu < c.basis.atom_norb[i]; ++mu)
            for (int nu = 0; nu < c.basis.atom_norb[j]; ++nu)
              e += 0.5 * w * pl(oi + mu, oj + nu) * (core.h(oi + mu, oj + nu) + fa(oi + mu, oj + nu));
        }
      so.energy = e;
    }

    // weighted spectra and the common Fermi level (:584-700)
    std::vector<std::vector<std::pair<double, double>>> spec(parts.size());
    for (size_t s = 0; s < parts.size(); ++s) {
      const Solution &so = sol[s];
      const int m = so.basis.nao;
      for (int ch = 0; ch < (uhf ? 2 : 1); ++ch) {
        const std::vector<double> &eps = ch ? so.eb : so.ea;
        const std::vector<double> &v = ch ? so.vb : so.va;
        const double scale = uhf ? 0.5 : 1.0;
        for (int k = 0; k < m; ++k) {
          double norm = 0.0;
          for (int i = 0; i < parts[s].n_core; ++i)
            for (int mu = 0; mu < so.basis.atom_norb[i]; ++mu) {
              const double c = v[(size_t)k * m + so.basis.atom_offset[i] + mu];
              norm += c * c;
            }
          spec[s].push_back({eps[k], scale * norm});
        }
      }
    }
    auto count = [&](double f) {
      double total = 0.0;
      for (const auto &st : spec) {
        double t = 0.0;
        for (const auto &ew : st) {
          const double occ = occupation(ew.first, f, dc.fermi_width_ev);
          t += occ < 1.0e-14 ? 0.0 : occ * ew.second;
        }
        total += t;
      }
      return total;
    };
    double lo = -500.0, hi = 500.0;
    if (count(lo) > n_elec || count(hi) < n_elec) {
      double a = INFINITY, b = -INFINITY;
      for (const Solution &so : sol)
        if (!so.ea.empty()) {
          a = std::min(a, so.ea.front());
          b = std::max(b, so.ea.back());
        }
      char buf[256];
      std::snprintf(buf, sizeof buf,
                    "no chemical potential in [-500, 500] eV holds %g electrons; the subsystem spectra span %.3f to "
                    "%.3f eV",
                    n_elec, a, b);
      throw Error(PM7_ERR_INVALID_INPUT, buf);
    }
    for (int it = 0; it < 200; ++it) {
      const double mid = 0.5 * (lo + hi);
      if (count(mid) < n_elec) lo = mid;
      else hi = mid;
      if (hi - lo < 1.0e-12) break;
    }
    fermi = 0.5 * (lo + hi);

    // reassembly (scatter_density, :770-814), normalisation, error and mixing
    Mat next(nao), next_s(nao);
    for (size_t s = 0; s < parts.size(); ++s) {
      const Solution &so = sol[s];
      const Part &pt = parts[s];
      const int m = so.basis.nao, n = (int)pt.parent.size();
      for (int spin = 0; spin < (uhf ? 2 : 1); ++spin) {
        Mat D(m);
        for (int ch = 0; ch < (uhf ? 2 : 1); ++ch) {
          const double scale = !uhf ? 1.0 : (ch == 0 ? 0.5 : (spin ? -0.5 : 0.5));
          const std::vector<double> &eps = ch ? so.eb : so.ea;
          const std::vector<double> &v = ch ? so.vb : so.va;
          for (int k = 0; k < m; ++k) {
            const double f = occupation(eps[k], fermi, dc.fermi_width_ev) * scale;
            if (std::fabs(f) < 1.0e-14) continue;
            const double *row = &v[(size_t)k * m];
            for (int a = 0; a < m; ++a)
              for (int b = 0; b < m; ++b) D(a, b) += f * row[a] * row[b];
          }
        }
        Mat &target = spin ? next_s : next;
        for (int i = 0; i < n; ++i)
          for (int j = 0; j < n; ++j) {
            const double w = pt.weight(i, j);
            if (w == 0.0) continue;
            const int gi = basis.atom_offset[pt.parent[i]], gj = basis.atom_offset[pt.parent[j]];
            const int li = so.basis.atom_offset[i], lj = so.basis.atom_offset[j];
            for (int mu = 0; mu < so.basis.atom_norb[i]; ++mu)
              for (int nu = 0; nu < so.basis.atom_norb[j]; ++nu) target(gi + mu, gj + nu) += w * D(li + mu, lj + nu);
          }
      }
    }
    double sq = 0.0;
    for (int k = 0; k < nao; ++k)
      for (int l = 0; l < nao; ++l) {
        const double wt = wtot[(size_t)basis.ao_atom[k] * N + basis.ao_atom[l]];
        if (!(wt > 0.0)) continue;
        const double norm = wt > 1.0e-12 ? 1.0 / wt : 0.0;
        const double nx = next(k, l) * norm;
        sq += (P(k, l) - nx) * (P(k, l) - nx);
        P(k, l) = (1.0 - dc.mixing) * P(k, l) + dc.mixing * nx;
        if (uhf) S(k, l) = (1.0 - dc.mixing) * S(k, l) + dc.mixing * (next_s(k, l) * norm);
      }
    err = std::sqrt(sq / (double)std::max<int64_t>(n_stored, 1));
    electronic = 0.0;
    for (const Solution &so : sol) electronic += so.energy;
    if (err < dc.p_tol) {
      converged = true;
      break;
    }
  }

  std::memset(r, 0, sizeof(*r));
  r->n_atoms = N;
  r->nao = nao;
  r->converged = converged ? 1 : 0;
  r->iterations = iterations;
  r->subsystems = (int)parts.size();
  r->largest_subsystem = largest_atoms;
  r->unrestricted = uhf ? 1 : 0;
  r->fermi_ev = fermi;
  r->electronic_ev = electronic;
  r->density_error = err;
  r->core_core_ev = core_core_energy(mol, p);
  double parts5[5];
  r->correction_ev = correction_energy(mol, o, parts5) * KCAL_TO_EV;
  r->energy_ev = electronic + r->core_core_ev + r->correction_ev;
  r->stored_density_elements = n_stored;
  const std::vector<double> pop = pops_of(P);
  r->charges = static_cast<double *>(std::malloc(sizeof(double) * std::max(N, 1)));
  for (int a = 0; a < N; ++a) r->charges[a] = cores[a] - pop[a];
  if (o.want_matrices) {
    r->density = static_cast<double *>(std::malloc(sizeof(double) * std::max<size_t>(P.a.size(), 1)));
    std::memcpy(r->density, P.a.data(), sizeof(double) * P.a.size());
    if (uhf) {
      r->spin_density = static_cast<double *>(std::malloc(sizeof(double) * std::max<size_t>(S.a.size(), 1)));
      std::memcpy(r->spin_density, S.a.data(), sizeof(double) * S.a.size());
    }
  }
}

}  // namespace
}  // namespace oracle

using namespace oracle;

extern "C" {

// The oracle's run_dandc (no gradient: the harness composes it from the fixed-density and
// correction gradients at the returned density).
pm7_status pm7_oracle_run_dandc(const pm7_molecule *m, const pm7_options *o, const pm7_dandc_options *dc,
                                pm7_dandc_result *r) {
  if (r) std::memset(r, 0, sizeof(*r));
  try {
    run_dandc(to_molecule(m), *o, *dc, r);
    g_error.clear();
    return PM7_OK;
  } catch (const Error &e) {
    g_error = e.what();
    return e.code;
  } catch (const std::exception &e) {
    g_error = e.what();
    return PM7_ERR_INVALID_INPUT;
  }
}

// The oracle's partition, in the layout of pm7_stage_dandc_partition.
pm7_status pm7_oracle_dandc_partition(const pm7_molecule *m, int32_t core_size, double buffer, int32_t *core_of,
                                      int32_t *sizes, int32_t *n_subsystems, int64_t *stored_pairs) {
  try {
    const Molecule mol = to_molecule(m);
    const std::vector<Part> parts = partition(mol, core_size, buffer);
    const int n = mol.size();
    std::vector<unsigned char> seen((size_t)n * n, 0);
    int64_t pairs = 0;
    for (size_t a = 0; a < parts.size(); ++a) {
      const Part &p = parts[a];
      sizes[a] = (int32_t)p.parent.size();
      for (int i = 0; i < p.n_core; ++i) core_of[p.parent[i]] = (int32_t)a;
      for (int i = 0; i < (int)p.parent.size(); ++i)
        for (int j = 0; j < (int)p.parent.size(); ++j)
          if (p.weight(i, j) > 0.0) {
            unsigned char &v = seen[(size_t)p.parent[i] * n + p.parent[j]];
            pairs += v == 0;
            v = 1;
          }
    }
    *n_subsystems = (int32_t)parts.size();
    *stored_pairs = pairs;
    return PM7_OK;
  } catch (const std::exception &e) {
    g_error = e.what();
    return PM7_ERR_INVALID_INPUT;
  }
}

void pm7_oracle_dandc_result_free(pm7_dandc_result *r) {
  if (!r) return;
  std::free(r->charges);
  std::free(r->gradient);
  std::free(r->density);
  std::free(r->spin_density);
  r->charges = r->gradient = r->density = r->spin_density = nullptr;
}

}  // extern "C"
