// Host-side control of the SCF loop: the extrapolation history bookkeeping and the
// stall guard. The dot products these need are computed on the device; what stays
// here is the <= 9x9 algebra of pm7-rs src/scf.rs:1534-1916.
#pragma once

#include <algorithm>
#include <cmath>
#include <limits>
#include <vector>

namespace pm7 {

// StallGuard (scf.rs:1581-1656): raises a level shift when two 5-iteration windows
// show neither a smaller density step nor a lower energy, relaxes it on fast progress.
struct StallGuardHost {
  double floor, shift;
  std::vector<double> steps, energies;
  explicit StallGuardHost(double f) : floor(f), shift(f) {}
  void update(double step, double energy) {
    const size_t W = 5;
    steps.push_back(step);
    energies.push_back(energy);
    const size_t n = steps.size();
    if (n < 2 * W) return;
    auto lowest = [](const std::vector<double> &v, size_t a, size_t b) {
      double m = std::numeric_limits<double>::infinity();
      for (size_t i = a; i < b; ++i) m = std::min(m, v[i]);
      return m;
    };
    const double s_now = lowest(steps, n - W, n), s_was = lowest(steps, n - 2 * W, n - W);
    const double e_now = lowest(energies, n - W, n), e_was = lowest(energies, n - 2 * W, n - W);
    bool moved = false;
    if (s_now <= s_was * 0.1) {
      if (shift > floor) {
        const double relaxed = std::max(shift * 0.5, floor);
        shift = relaxed < 0.25 ? floor : relaxed;
        moved = true;
      }
    } else if (s_now > s_was * 0.9 && e_now > e_was - 1.0e-9 && shift < 64.0) {
      shift = shift < 1.0 ? 1.0 : std::min(shift * 2.0, 64.0);
      moved = true;
    }
    if (moved) {
      steps.clear();
      energies.clear();
    } else {
      steps.erase(steps.begin());
      energies.erase(energies.begin());
    }
  }
};

// Ring of at most `kmax` (F, [F,P], D) triples in device memory, tracked here in
// chronological order together with the cached inner products <e_i, e_j> and
// <D_i, F_j>. Each iteration adds one row/column of each, so nothing is recomputed.
class HistoryHost {
 public:
  explicit HistoryHost(int kmax) : kmax_(kmax), gram_(kmax * kmax, 0.0), xdf_(kmax * kmax, 0.0) {}

  // Make room for a new entry; returns its slot. The returned slot is the newest.
  int push() {
    int slot;
    if ((int)order_.size() < kmax_) {
      slot = (int)order_.size();
    } else {
      slot = order_.front();
      order_.erase(order_.begin());
    }
    pending_ = slot;
    return slot;
  }
  // Older entries (chronological, oldest first), excluding the newest.
  const std::vector<int> &order() const { return order_; }

  // ee[i] = <e_i, e_new> for older i plus <e_new, e_new> last; df_row[j] = <D_new, F_j>
  // for older j plus <D_new, F_new> last; df_col[i] = <D_i, F_new> for older i.
  void record(const std::vector<double> &ee, const std::vector<double> &df_row, const std::vector<double> &df_col) {
    const int s = pending_;
    const size_t k = order_.size();
    for (size_t i = 0; i < k; ++i) {
      const int o = order_[i];
      gram_[o * kmax_ + s] = gram_[s * kmax_ + o] = ee[i];
      xdf_[s * kmax_ + o] = df_row[i];
      xdf_[o * kmax_ + s] = df_col[i];
    }
    gram_[s * kmax_ + s] = ee[k];
    xdf_[s * kmax_ + s] = df_row[k];
    order_.push_back(s);
  }
  const std::vector<int> &entries() const { return order_; }

  // CDIIS weights over the chronological entries (scf.rs:1684-1806); empty = fall back.
  std::vector<double> cdiis() const {
    const int n = (int)order_.size();
    if (n < 2) return {};
    for (int skip = 0; skip + 1 < n; ++skip) {
      const int m = n - skip;
      if (m < 2) continue;
      double scale = 0.0;
      for (int i = 0; i < m; ++i) scale = std::max(scale, std::fabs(g(skip + i, skip + i)));
      if (!std::isfinite(scale) || scale <= 0.0) continue;
      const int dim = m + 1;
      std::vector<double> b(dim * dim, 0.0), rhs(dim, 0.0), c;
      for (int i = 0; i < m; ++i) {
        for (int j = 0; j < m; ++j) b[i * dim + j] = g(skip + i, skip + j) / scale;
        b[i * dim + m] = -1.0;
        b[m * dim + i] = -1.0;
      }
      rhs[m] = -1.0;
      if (!solve(b, dim, rhs, c)) continue;
      bool finite = true;
      for (double v : c) finite = finite && std::isfinite(v);
      if (!finite) continue;
      double wsum = 0.0;
      for (int i = 0; i < m; ++i) wsum += std::fabs(c[i]);
      if (wsum <= 25.0) {
        std::vector<double> w(n, 0.0);
        for (int i = 0; i < m; ++i) w[skip + i] = c[i];
        return w;
      }
    }
    return {};
  }

  // A-DIIS weights (scf.rs:1812-1916): projected gradient on the simplex.
  std::vector<double> adiis() const {
    const int n = (int)order_.size();
    if (n < 2) return {};
    const int last = n - 1;
    std::vector<double> d(n), s(n * n);
    for (int i = 0; i < n; ++i) {
      d[i] = x(i, last) - x(last, last);
      for (int j = 0; j < n; ++j) s[i * n + j] = x(i, j) - x(i, last) - x(last, j) + x(last, last);
    }
    double l = 1.0e-12;
    for (int i = 0; i < n; ++i) {
      double row = 0.0;
      for (int j = 0; j < n; ++j) row += std::fabs(s[i * n + j] + s[j * n + i]);
      l = std::max(l, row);
    }
    const double lr = 1.0 / l;
    std::vector<double> c(n, 0.0), gr(n), trial(n);
    c[last] = 1.0;
    for (int it = 0; it < 400; ++it) {
      for (int k = 0; k < n; ++k) {
        double acc = 2.0 * d[k];
        for (int j = 0; j < n; ++j) acc += (s[k * n + j] + s[j * n + k]) * c[j];
        gr[k] = acc;
      }
      for (int i = 0; i < n; ++i) trial[i] = c[i] - lr * gr[i];
      std::vector<double> proj = project(trial);
      double delta = 0.0;
      for (int i = 0; i < n; ++i) delta += std::fabs(proj[i] - c[i]);
      c = proj;
      if (delta < 1.0e-12) break;
    }
    return c;
  }

 private:
  double g(int i, int j) const { return gram_[order_[i] * kmax_ + order_[j]]; }
  double x(int i, int j) const { return xdf_[order_[i] * kmax_ + order_[j]]; }

  static std::vector<double> project(const std::vector<double> &v) {
    std::vector<double> u = v;
    std::sort(u.begin(), u.end(), [](double a, double b) { return a > b; });
    double css = 0.0, theta = 0.0;
    for (size_t j = 0; j < u.size(); ++j) {
      css += u[j];
      const double t = (css - 1.0) / (j + 1.0);
      if (u[j] - t > 0.0) theta = t;
    }
    std::vector<double> out(v.size());
    for (size_t i = 0; i < v.size(); ++i) out[i] = std::max(v[i] - theta, 0.0);
    return out;
  }

  // Gaussian elimination with partial pivoting; false when (near-)singular.
  static bool solve(std::vector<double> m, int n, std::vector<double> rhs, std::vector<double> &x) {
    for (int col = 0; col < n; ++col) {
      int piv = col;
      double best = std::fabs(m[col * n + col]);
      for (int r = col + 1; r < n; ++r)
        if (std::fabs(m[r * n + col]) > best) {
          best = std::fabs(m[r * n + col]);
          piv = r;
        }
      if (best < 1.0e-12) return false;
      if (piv != col) {
        for (int j = 0; j < n; ++j) std::swap(m[col * n + j], m[piv * n + j]);
        std::swap(rhs[col], rhs[piv]);
      }
      for (int r = col + 1; r < n; ++r) {
        const double f = m[r * n + col] / m[col * n + col];
        if (f == 0.0) continue;
        for (int j = col; j < n; ++j) m[r * n + j] -= f * m[col * n + j];
        rhs[r] -= f * rhs[col];
      }
    }
    x.assign(n, 0.0);
    for (int col = n - 1; col >= 0; --col) {
      double s = rhs[col];
      for (int j = col + 1; j < n; ++j) s -= m[col * n + j] * x[j];
      x[col] = s / m[col * n + col];
    }
    return true;
  }

  int kmax_;
  std::vector<int> order_;
  int pending_ = 0;
  std::vector<double> gram_, xdf_;
};

}  // namespace pm7
