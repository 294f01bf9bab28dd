// Host-side plan construction: the footprint tables every engine reads, built once per
// (grid, kernel, scale, mask strategy) as Filtering.plan_filter does (Filtering.jl:2931-2954).
// Geometry follows the reference's documented conventions: great-circle distance in the
// haversine form (Filtering.jl:264-265), cell measure R^2 cos(phi) dlambda dphi
// (docs/src/theory.md:307), kernel weights and radii of Kernels.jl:318-379.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <numeric>
#include <thread>

#include "cgef_internal.h"

namespace cgef {

double kernel_weight(int kernel, double alpha, double d, double ell) {
  if (kernel == CGEF_TOPHAT) return d <= ell / 2.0 ? 1.0 : 0.0;  // Kernels.jl:318-320
  double q = d / ell;
  return std::exp(-alpha * (q * q));  // Kernels.jl:322-324
}

double kernel_radius(int kernel, double alpha, double ell) {
  if (kernel == CGEF_TOPHAT) return ell / 2.0;                       // Kernels.jl:354
  return ell * std::sqrt(-std::log(kGaussianTruncationTol) / alpha);  // Kernels.jl:356-359
}

namespace {

inline double coord(double x0, double d, int i) { return std::fma(static_cast<double>(i), d, x0); }

// Column half-width that certainly covers the part of row phi2 within rad of (0, phi1): the
// spherical band formula plus a two-cell margin, capped at `cap`.  Inclusion itself is decided by
// the distance test, so only coverage matters here.
int sphere_row_window(double R, double dx, double phi1, double phi2, double rad, int cap) {
  double den = std::cos(phi1) * std::cos(phi2);
  double num = std::cos(rad / R) - std::sin(phi1) * std::sin(phi2);
  if (den <= 0.0) return cap;
  double c = num / den;
  if (c <= -1.0) return cap;
  if (c > 1.0) return std::min(2, cap);
  double w = std::floor(std::acos(c) / std::fabs(dx)) + 2.0;
  return w > cap ? cap : static_cast<int>(w);
}

// Connectivity.metric_band (Filtering.jl:761-765, 1004): axis-1 half-width of the top-hat
// support between rows y_t and y_s, negative when the row is out of reach.
double metric_band(int geometry, double R, double y_t, double y_s, double rad) {
  if (geometry == CGEF_CARTESIAN) {
    double dy = y_s - y_t;
    double r2 = rad * rad - dy * dy;
    return r2 < 0.0 ? -1.0 : std::sqrt(r2);
  }
  double den = std::cos(y_t) * std::cos(y_s);
  double num = std::cos(rad / R) - std::sin(y_t) * std::sin(y_s);
  if (den <= 0.0) return num <= 0.0 ? M_PI : -1.0;
  double c = num / den;
  if (c > 1.0) return -1.0;
  if (c < -1.0) return M_PI;
  return std::acos(c);
}

// Runs body(i) for i in [0, n) on the host's cores (results must not depend on the order).
template <typename F>
void parallel_for(int n, F body) {
  unsigned hw = std::thread::hardware_concurrency();
  int nt = static_cast<int>(std::min<unsigned>(hw == 0 ? 1 : hw, 32));
  if (nt <= 1 || n < 64) {
    for (int i = 0; i < n; ++i) body(i);
    return;
  }
  std::atomic<int> next{0};
  std::vector<std::thread> pool;
  for (int t = 0; t < nt; ++t)
    pool.emplace_back([&]() {
      for (int i = next.fetch_add(1); i < n; i = next.fetch_add(1)) body(i);
    });
  for (auto& th : pool) th.join();
}

template <typename T>
int upload(const cgef_plan* p, T** dst, const T* src, size_t n) {
  if (n == 0 || p->device < 0) {  // no device: host tables only
    *dst = nullptr;
    return CGEF_OK;
  }
  cudaError_t e = cudaMalloc(reinterpret_cast<void**>(dst), n * sizeof(T));
  if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(plan table)");
  e = cudaMemcpy(*dst, src, n * sizeof(T), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpy(plan table)");
  return CGEF_OK;
}

struct Banded {
  int D = 0;
  int Amax = 0;
  std::vector<BandRow> rows;  // ny * (2D+1) (sphere) or 2D+1 (Cartesian, one band)
  std::vector<double> w;      // half rows
  std::vector<int64_t> ptr;   // CSR band offsets (entry counts of the reference's layout)
};

// Banded footprint (Filtering.jl:636-732).  Each (band, row offset) holds a contiguous
// longitude interval [-a, hi]; weights are stored once per |di| because the kernel of the
// great-circle (or Euclidean) distance is even in di.  A column inside the interval that fails
// d <= rad keeps weight 0, which adds nothing to either sum of finite values, so the entry set is the
// reference's (a slice holding a non-finite value is summed with zero weights skipped).
int build_banded(const cgef_plan* p, Banded& B) {
  const int nx = p->nx, ny = p->ny;
  const double rad = p->rad;
  const bool sphere = p->geometry == CGEF_SPHERICAL;
  if (!sphere) {
    const double cells_x = p->dx > 0 ? std::ceil(rad / p->dx) : 0.0;
    const double cells_y = p->dy > 0 ? std::ceil(rad / p->dy) : 0.0;
    if ((2.0 * cells_y + 1.0) * (cells_x + 1.0) > static_cast<double>(INT32_MAX))
      return fail(CGEF_EINVAL, "footprint too large: more than 2^31 half-row weights (reduce the scale or the grid)");
    const int di_lim = static_cast<int>(cells_x);
    const int dj_lim = static_cast<int>(cells_y);
    const double A = p->dx * p->dy;
    B.D = dj_lim;
    B.rows.assign(2 * dj_lim + 1, BandRow{0, -1, -1, 0});
    B.ptr.push_back(0);
    int64_t n = 0;
    for (int ddj = -dj_lim; ddj <= dj_lim; ++ddj) {
      int a = -1;
      for (int ddi = 0; ddi <= di_lim; ++ddi) {
        double x = ddi * p->dx, y = ddj * p->dy;
        double d = std::sqrt(x * x + y * y);
        if (d <= rad) a = ddi;
      }
      BandRow& r = B.rows[ddj + dj_lim];
      if (a >= 0) {
        r.woff = static_cast<int32_t>(B.w.size());
        r.a = a;
        r.hi = a;
        for (int ddi = 0; ddi <= a; ++ddi) {
          double x = ddi * p->dx, y = ddj * p->dy;
          double d = std::sqrt(x * x + y * y);
          B.w.push_back(d <= rad ? kernel_weight(p->kernel, p->alpha, d, p->scale) * A : 0.0);
          if (d <= rad) n += ddi == 0 ? 1 : 2;
        }
        B.Amax = std::max(B.Amax, a);
      }
    }
    B.ptr.push_back(n);
    return CGEF_OK;
  }
  const int dj_lim = p->dy > 0 ? static_cast<int>(std::ceil(rad / (p->R * p->dy))) : 0;
  const int half = nx / 2;
  B.D = dj_lim;
  B.rows.assign(static_cast<size_t>(ny) * (2 * dj_lim + 1), BandRow{0, -1, -1, 0});
  // every band is built independently (in parallel), then concatenated in band order
  struct BandOut {
    std::vector<double> whalf;
    std::vector<int32_t> a, hi, off;  // per row offset, off relative to the band's whalf
    int64_t n = 0;                    // entries (d <= rad) of the band
  };
  std::vector<BandOut> outs(ny);
  parallel_for(ny, [&](int j) {
    BandOut& o = outs[j];
    o.a.assign(2 * dj_lim + 1, -1);
    o.hi.assign(2 * dj_lim + 1, -1);
    o.off.assign(2 * dj_lim + 1, 0);
    const double phi = coord(p->y0, p->dy, j);
    bool closed = false;
    for (int ddj = -dj_lim; ddj <= dj_lim; ++ddj) {
      int jj = j + ddj;
      if (jj < 0 || jj >= ny) continue;
      if (sphere_row_window(p->R, p->dx, phi, coord(p->y0, p->dy, jj), rad, half) >= half) closed = true;
    }
    for (int ddj = -dj_lim; ddj <= dj_lim; ++ddj) {
      int jj = j + ddj;
      if (jj < 0 || jj >= ny) continue;
      const double phi2 = coord(p->y0, p->dy, jj);
      const double A = p->R * p->R * std::cos(phi2) * p->dx * p->dy;
      const int win = closed ? half : sphere_row_window(p->R, p->dx, phi, phi2, rad, half);
      // the reference visits ddi in [-win, hi]; hi = half - 1 where the ring closes on an even nx
      // (column -half is column +half)
      const int hi = (closed && 2 * half + 1 > nx) ? half - 1 : win;
      // weights by |di|; inclusion exactly as the reference (d <= rad at each visited offset).  The
      // great-circle distance from (0, phi) to (ddi dx, phi2) in the haversine form,
      //     d = 2 R asin(sqrt(min(1, sin^2((phi2 - phi) / 2) + cos(phi) cos(phi2) sin^2(ddi dx / 2)))),
      // with its row-constant factors computed once; it is even in ddi bit for bit (sin is odd), so
      // each |ddi| is evaluated once and counted for every visited sign.
      const double sdp = std::sin((phi2 - phi) / 2.0);
      const double cc = std::cos(phi) * std::cos(phi2);
      int amax = -1;
      std::vector<double> wabs(static_cast<size_t>(win) + 1, 0.0);
      for (int k = 0; k <= win; ++k) {
        const double sdl = std::sin((static_cast<double>(k) * p->dx - 0.0) / 2.0);
        double h = sdp * sdp + cc * sdl * sdl;
        if (h > 1.0) h = 1.0;
        const double d = 2.0 * p->R * std::asin(std::sqrt(h));
        if (d <= rad) {
          wabs[k] = kernel_weight(p->kernel, p->alpha, d, p->scale) * A;
          amax = k;
          o.n += k == 0 ? 1 : 1 + (k <= hi ? 1 : 0);  // -k always visited, +k up to hi
        }
      }
      if (amax >= 0) {
        const int r = ddj + dj_lim;
        o.off[r] = static_cast<int32_t>(o.whalf.size());
        o.a[r] = amax;
        o.hi[r] = std::min(amax, hi);
        for (int k = 0; k <= amax; ++k) o.whalf.push_back(wabs[k]);
      }
    }
  });
  // concatenate in band order: each band's half rows go to its offset in one pre-sized array
  std::vector<size_t> base(static_cast<size_t>(ny) + 1, 0);
  for (int j = 0; j < ny; ++j) base[j + 1] = base[j] + outs[j].whalf.size();
  // the half rows are indexed by 32-bit offsets (BandRow::woff): refuse before sizing the table
  if (base[ny] > static_cast<size_t>(INT32_MAX))
    return fail(CGEF_EINVAL, "footprint too large: more than 2^31 half-row weights (reduce the scale or the grid)");
  B.w.resize(base[ny]);
  parallel_for(ny, [&](int j) {
    BandOut& o = outs[j];
    std::copy(o.whalf.begin(), o.whalf.end(), B.w.begin() + static_cast<std::ptrdiff_t>(base[j]));
    for (int r = 0; r < 2 * dj_lim + 1; ++r) {
      BandRow& br = B.rows[static_cast<size_t>(j) * (2 * dj_lim + 1) + r];
      if (o.a[r] >= 0) {
        br.woff = static_cast<int32_t>(base[j]) + o.off[r];
        br.a = o.a[r];
        br.hi = o.hi[r];
      }
    }
    std::vector<double>().swap(o.whalf);
  });
  B.ptr.push_back(0);
  for (int j = 0; j < ny; ++j) {
    for (int a : outs[j].a) B.Amax = std::max(B.Amax, a);
    B.ptr.push_back(B.ptr.back() + outs[j].n);
  }
  return CGEF_OK;
}

// Rows of the spherical banded footprint for the device build (device_band_tables): every inclusion
// decided here with libm, the weights left to the device.  Per (band, row offset), h -- and so the
// distance -- grows with |di| over [0, half] (sin^2 increases there and cos(phi) cos(phi') >= 0), so the
// included offsets are |di| <= a; a is found by bisection over the row's window, then the offsets within
// four of it are tested one by one, and a row where rounding breaks the order there is built entirely
// here, as build_banded does, zero weights included.  The rows and entry counts are build_banded's.
struct DeviceRows {
  std::vector<double> sdp, cc, area;  // per band row: sin((phi' - phi) / 2), cos(phi) cos(phi'), cell measure
  std::vector<double> sdl;            // sin(k dlambda / 2), k <= nx / 2
  std::vector<std::pair<int64_t, std::vector<double>>> host_rows;  // (woff, weights) built here
  size_t nweights = 0;
};

int build_banded_sphere_rows(const cgef_plan* p, Banded& B, DeviceRows& dr) {
  const int nx = p->nx, ny = p->ny;
  const double rad = p->rad;
  const int dj_lim = p->dy > 0 ? static_cast<int>(std::ceil(rad / (p->R * p->dy))) : 0;
  const int half = nx / 2;
  const int W = 2 * dj_lim + 1;
  B.D = dj_lim;
  B.rows.assign(static_cast<size_t>(ny) * W, BandRow{0, -1, -1, 0});
  dr.sdp.assign(static_cast<size_t>(ny) * W, 0.0);
  dr.cc.assign(static_cast<size_t>(ny) * W, 0.0);
  dr.area.assign(static_cast<size_t>(ny) * W, 0.0);
  dr.sdl.resize(static_cast<size_t>(half) + 1);
  for (int k = 0; k <= half; ++k) dr.sdl[k] = std::sin((static_cast<double>(k) * p->dx - 0.0) / 2.0);
  std::vector<int64_t> counts(ny, 0);
  std::vector<std::vector<std::pair<int, std::vector<double>>>> own(ny);  // per band: (row, weights)
  parallel_for(ny, [&](int j) {
    const double phi = coord(p->y0, p->dy, j);
    bool closed = false;
    for (int ddj = -dj_lim; ddj <= dj_lim; ++ddj) {
      int jj = j + ddj;
      if (jj < 0 || jj >= ny) continue;
      if (sphere_row_window(p->R, p->dx, phi, coord(p->y0, p->dy, jj), rad, half) >= half) closed = true;
    }
    for (int ddj = -dj_lim; ddj <= dj_lim; ++ddj) {
      int jj = j + ddj;
      if (jj < 0 || jj >= ny) continue;
      const size_t r = static_cast<size_t>(j) * W + (ddj + dj_lim);
      const double phi2 = coord(p->y0, p->dy, jj);
      const double A = p->R * p->R * std::cos(phi2) * p->dx * p->dy;
      const int win = closed ? half : sphere_row_window(p->R, p->dx, phi, phi2, rad, half);
      const int hi = (closed && 2 * half + 1 > nx) ? half - 1 : win;
      const double sdp = std::sin((phi2 - phi) / 2.0);
      const double cc = std::cos(phi) * std::cos(phi2);
      auto dist = [&](int k) {
        const double sdl = dr.sdl[k];
        double h = sdp * sdp + cc * sdl * sdl;
        if (h > 1.0) h = 1.0;
        return 2.0 * p->R * std::asin(std::sqrt(h));
      };
      int amax = -1;
      if (dist(0) <= rad) {
        int lo = 0, up = win;
        while (lo < up) {
          const int mid = lo + (up - lo + 1) / 2;
          if (dist(mid) <= rad)
            lo = mid;
          else
            up = mid - 1;
        }
        amax = lo;
      }
      bool monotone = true;
      for (int k = std::max(0, amax - 4); k <= std::min(win, amax + 4) && monotone; ++k)
        monotone = (dist(k) <= rad) == (k <= amax);
      if (!monotone) {
        // build_banded's loop over the whole window: inclusion per offset, zero weights in the gaps
        std::vector<double> wabs(static_cast<size_t>(win) + 1, 0.0);
        amax = -1;
        int64_t n = 0;
        for (int k = 0; k <= win; ++k) {
          const double d = dist(k);
          if (d <= rad) {
            wabs[k] = kernel_weight(p->kernel, p->alpha, d, p->scale) * A;
            amax = k;
            n += k == 0 ? 1 : 1 + (k <= hi ? 1 : 0);
          }
        }
        counts[j] += n;
        if (amax >= 0) {
          wabs.resize(static_cast<size_t>(amax) + 1);
          own[j].emplace_back(ddj + dj_lim, std::move(wabs));
        }
      } else if (amax >= 0) {
        counts[j] += 1 + amax + std::min(amax, hi);
      }
      if (amax >= 0) {
        BandRow& br = B.rows[r];
        br.a = amax;
        br.hi = std::min(amax, hi);
        dr.sdp[r] = sdp;
        dr.cc[r] = cc;
        dr.area[r] = A;
      }
    }
  });
  // half-row offsets in band order, then the entry counts of the reference's CSR
  size_t off = 0;
  for (size_t r = 0; r < B.rows.size(); ++r) {
    BandRow& br = B.rows[r];
    if (br.a < 0) continue;
    if (off > static_cast<size_t>(INT32_MAX))
      return fail(CGEF_EINVAL, "footprint too large: more than 2^31 half-row weights (reduce the scale or the grid)");
    br.woff = static_cast<int32_t>(off);
    off += static_cast<size_t>(br.a) + 1;
    B.Amax = std::max(B.Amax, br.a);
  }
  if (off > static_cast<size_t>(INT32_MAX))
    return fail(CGEF_EINVAL, "footprint too large: more than 2^31 half-row weights (reduce the scale or the grid)");
  dr.nweights = off;
  for (int j = 0; j < ny; ++j)
    for (auto& rw : own[j])
      dr.host_rows.emplace_back(B.rows[static_cast<size_t>(j) * W + rw.first].woff, std::move(rw.second));
  B.ptr.assign(1, 0);
  for (int j = 0; j < ny; ++j) B.ptr.push_back(B.ptr.back() + counts[j]);
  return CGEF_OK;
}

// Process-wide choice of where large spherical footprints are built (cgef_set_footprint_build).
std::atomic<int> g_footprint_build{CGEF_BUILD_AUTO};

// The device build applies to the banded engine on a sphere with a periodic longitude (one ZeroFill
// denominator per band) and a device; AUTO takes it once the footprint holds about 2e6 half-row weights,
// where the host's distance loop starts to cost tens of milliseconds.
bool use_device_build(const cgef_plan* p) {
  if (p->engine != CGEF_ENGINE_BANDED || p->geometry != CGEF_SPHERICAL || !p->periodic_x || p->device < 0) return false;
  const int mode = g_footprint_build.load();
  if (mode == CGEF_BUILD_HOST) return false;
  if (mode == CGEF_BUILD_DEVICE) return true;
  const int dj_lim = p->dy > 0 ? static_cast<int>(std::ceil(p->rad / (p->R * p->dy))) : 0;
  double est = 0.0;
  for (int j = 0; j < p->ny; ++j) {
    const double c = std::fabs(std::cos(coord(p->y0, p->dy, j)));
    const double cells = c > 0.0 ? p->rad / (p->R * c * p->dx) : p->nx / 2.0;
    est += (2.0 * dj_lim + 1.0) * (std::min(cells, p->nx / 2.0) + 1.0);
  }
  return est > 2e6;
}

}  // namespace

int set_footprint_build(int where) {
  if (where != CGEF_BUILD_AUTO && where != CGEF_BUILD_HOST && where != CGEF_BUILD_DEVICE)
    return fail(CGEF_EINVAL, "footprint build must be CGEF_BUILD_AUTO, CGEF_BUILD_HOST or CGEF_BUILD_DEVICE");
  g_footprint_build.store(where);
  return CGEF_OK;
}

#ifndef CGEF_PAIRED
#define CGEF_PAIRED 1
#endif
#ifndef CGEF_SPLIT_WAVES
#define CGEF_SPLIT_WAVES 4.0
#endif

std::vector<double> group_row_costs(const cgef_plan* p, int j0, int R) {
  const bool sphere = p->geometry == CGEF_SPHERICAL;
  const int W = 2 * p->D + 1;
  std::vector<double> rc;
  rc.reserve(R + 2 * p->D);
  for (int jr = j0 - p->D; jr <= j0 + R - 1 + p->D; ++jr) {
    double c = 0.0;
    if (p->periodic_y || (jr >= 0 && jr < p->ny)) {
      int A = -1, HI = -1;
      for (int t = 0; t < R; ++t) {
        const int j = j0 + t;
        if (j >= p->ny) continue;
        const int dj = jr - j;
        if (dj < -p->D || dj > p->D) continue;
        const BandRow& r = p->h_rows[(sphere ? static_cast<size_t>(j) * W : 0) + (dj + p->D)];
        A = std::max(A, r.a);
        HI = std::max(HI, r.hi);
      }
      if (A >= 0) c = static_cast<double>(HI + A + 1) + 4.0;  // + per-row overhead
    }
    rc.push_back(c);
  }
  return rc;
}

void emit_group_items(int x0, int j0, int D, const std::vector<double>& rc, double target, std::vector<WorkItem>& items,
                      std::vector<SplitGroup>& groups, int& slots) {
  const int jlo = j0 - D;
  double cg = 0.0;
  for (double c : rc) cg += c;
  if (cg <= 0.0) {
    items.push_back(WorkItem{x0, j0, jlo, jlo, -1, 0});
    return;
  }
  const int nrow = static_cast<int>(rc.size());
  const int nsplit = std::max(1, std::min(nrow, static_cast<int>(std::ceil(cg / target))));
  // contiguous source-row parts of about equal cost
  std::vector<int> cut{0};
  double acc = 0.0;
  for (int r = 0; r < nrow; ++r) {
    acc += rc[r];
    if (static_cast<int>(cut.size()) < nsplit && acc >= cg * cut.size() / nsplit && r + 1 < nrow) cut.push_back(r + 1);
  }
  cut.push_back(nrow);
  const int parts = static_cast<int>(cut.size()) - 1;
  if (parts == 1) {
    items.push_back(WorkItem{x0, j0, jlo, jlo + cut[1], -1, static_cast<int32_t>(std::min(cg, 2e9))});
    return;
  }
  groups.push_back(SplitGroup{x0, j0, slots, parts});
  for (int q = 0; q < parts; ++q) {
    double c = 0.0;
    for (int r = cut[q]; r < cut[q + 1]; ++r) c += rc[r];
    items.push_back(WorkItem{x0, j0, jlo + cut[q], jlo + cut[q + 1], slots + q, static_cast<int32_t>(std::min(c, 2e9))});
  }
  slots += parts;
}

void subset_schedule(const cgef_plan* p, const std::vector<std::pair<int, int>>& tiles, int sms,
                     std::vector<WorkItem>& items, std::vector<SplitGroup>& groups, int& slots) {
  struct G {
    int x0, j0;
    std::vector<double> rc;
  };
  std::vector<G> gs;
  double total = 0.0;
  for (const auto& t : tiles)
    for (int r = 0; r < 32; r += kRows) {
      const int j0 = t.second * 32 + r;
      if (j0 >= p->ny) break;
      gs.push_back(G{t.first * 32, j0, group_row_costs(p, j0)});
      for (double c : gs.back().rc) total += c;
    }
  const double target = std::max(64.0, total / (sms * 16.0));
  items.clear();
  groups.clear();
  slots = 0;
  for (const G& g : gs) emit_group_items(g.x0, g.j0, p->D, g.rc, target, items, groups, slots);
  std::stable_sort(items.begin(), items.end(), [](const WorkItem& a, const WorkItem& b) { return a.cost > b.cost; });
}

int rebuild_schedule(cgef_plan* p, double waves, int which) {
  if (!(waves > 0.0)) return fail(CGEF_EINVAL, "split waves must be positive");
  if (which < 0 || which > 1) return fail(CGEF_EINVAL, "schedule index must be 0 or 1");
  Schedule& S = p->sched[which];
  const int R = which == 0 ? kRows : kRowsTall;
  if (S.rowcost.empty()) {
    const int ngroups = (p->ny + R - 1) / R;
    S.rowcost.assign(ngroups, {});
    parallel_for(ngroups, [&](int g) { S.rowcost[g] = group_row_costs(p, g * R, R); });
  }
  const int ngroups = static_cast<int>(S.rowcost.size());
  double total = 0.0;
  const int ntx = (p->nx + 31) / 32;
  for (int g = 0; g < ngroups; ++g)
    for (double c : S.rowcost[g]) total += c * ntx;
  int sms = 148;
  {
    int dev = 0;
    cudaDeviceProp prop;
    if (p->device >= 0 && cudaGetDevice(&dev) == cudaSuccess && cudaGetDeviceProperties(&prop, dev) == cudaSuccess)
      sms = prop.multiProcessorCount;
    else
      cudaGetLastError();
  }
  // about `waves` rounds of 16 resident warps per SM
  const double target = std::max(64.0, total / (sms * 16.0 * waves));
  std::vector<WorkItem> items;
  std::vector<SplitGroup> groups;
  int slots = 0;
  for (int g = 0; g < ngroups; ++g)
    for (int x = 0; x < p->nx; x += 32) emit_group_items(x, g * R, p->D, S.rowcost[g], target, items, groups, slots);
  std::stable_sort(items.begin(), items.end(), [](const WorkItem& a, const WorkItem& b) { return a.cost > b.cost; });
  if (S.d_items) cudaFree(S.d_items);
  if (S.d_groups) cudaFree(S.d_groups);
  S.d_items = nullptr;
  S.d_groups = nullptr;
  S.h_items = std::move(items);
  S.h_groups = std::move(groups);
  S.nslots = slots;
  S.waves = waves;
  S.rows = R;
  int rc;
  if ((rc = upload(p, &S.d_items, S.h_items.data(), S.h_items.size())) != CGEF_OK) return rc;
  return upload(p, &S.d_groups, S.h_groups.data(), S.h_groups.size());
}

int build_plan_tables(cgef_plan* p) {
  const int nx = p->nx, ny = p->ny;
  const bool sphere = p->geometry == CGEF_SPHERICAL;
  p->rad = kernel_radius(p->kernel, p->alpha, p->scale);
  p->h_x.resize(nx);
  p->h_y.resize(ny);
  for (int i = 0; i < nx; ++i) p->h_x[i] = coord(p->x0, p->dx, i);
  for (int j = 0; j < ny; ++j) p->h_y[j] = coord(p->y0, p->dy, j);
  std::vector<double> sinlam(nx), coslam(nx), sinphi(ny), cosphi(ny), area(ny), xscale(ny), tanfac(ny);
  for (int i = 0; i < nx; ++i) {
    sinlam[i] = std::sin(p->h_x[i]);
    coslam[i] = std::cos(p->h_x[i]);
  }
  for (int j = 0; j < ny; ++j) {
    double phi = p->h_y[j];
    sinphi[j] = std::sin(phi);
    cosphi[j] = std::cos(phi);
    if (sphere) {
      area[j] = p->R * p->R * std::cos(phi) * p->dx * p->dy;
      double c = std::cos(phi);
      xscale[j] = std::fabs(c) < std::sqrt(2.220446049250313e-16) ? 0.0 : 1.0 / (p->R * c);
      double sp = std::sin(phi), cp = std::cos(phi);
      tanfac[j] = std::fabs(cp) > 1e-12 ? sp / (p->R * cp) : 0.0;
    } else {
      area[j] = p->dx * p->dy;
      xscale[j] = 1.0;
      tanfac[j] = 0.0;
    }
  }
  p->active_area = 0.0;
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i)
      if (p->h_mask.empty() || p->h_mask[static_cast<size_t>(j) * nx + i]) p->active_area += area[j];

  Banded B;
  std::vector<double> den_zf;
  std::vector<double> gx, gy, px, py;
  std::vector<double> xe, prefix_wx;
  std::vector<PrefixRow> prows;

  if (p->engine == CGEF_ENGINE_BANDED) {
    const bool on_device = use_device_build(p);
    DeviceRows dr;
    if (int rc = on_device ? build_banded_sphere_rows(p, B, dr) : build_banded(p, B)) return rc;
    p->built_on_device = on_device;
    p->nwhalf = on_device ? static_cast<int64_t>(dr.nweights) : static_cast<int64_t>(B.w.size());
    p->D = B.D;
    p->Amax = B.Amax;
    p->dj_lim = B.D;
    p->di_max = B.Amax;
    p->h_rows = std::move(B.rows);
    p->h_whalf = std::move(B.w);
    p->h_ptr = std::move(B.ptr);
    p->nentries = p->h_ptr.back();
    // ZeroFill denominator: the footprint mass over in-domain entries, in CSR order
    // (Filtering.jl:2574-2582 accumulate w for every in-domain entry).
    const int64_t W = 2 * B.D + 1;
    if (on_device) {
      // the denominators come from the device weights (device_band_tables)
    } else if (p->periodic_x) {
      p->den_zf_2d = 0;
      den_zf.assign(ny, 0.0);
      parallel_for(ny, [&](int j) {
        double s = 0.0;
        for_each_entry(p, sphere ? j : 0, [&](int, int ddj, double w) {
          int jj = j + ddj;
          if ((jj < 0 || jj >= ny) && !p->periodic_y) return;
          s += w;
        });
        den_zf[j] = s;
      });
    } else {
      p->den_zf_2d = 1;
      den_zf.assign(static_cast<size_t>(ny) * nx, 0.0);
      parallel_for(ny, [&](int j) {
        const int b = sphere ? j : 0;
        // interior columns see every entry; edge columns are summed entry by entry
        double full = 0.0;
        for_each_entry(p, b, [&](int, int ddj, double w) {
          int jj = j + ddj;
          if ((jj < 0 || jj >= ny) && !p->periodic_y) return;
          full += w;
        });
        for (int i = 0; i < nx; ++i) {
          double s = full;
          if (i < B.Amax || i >= nx - B.Amax) {
            s = 0.0;
            for_each_entry(p, b, [&](int ddi, int ddj, double w) {
              int jj = j + ddj;
              if ((jj < 0 || jj >= ny) && !p->periodic_y) return;
              int ii = i + ddi;
              if (ii < 0 || ii >= nx) return;
              s += w;
            });
          }
          den_zf[static_cast<size_t>(j) * nx + i] = s;
        }
      });
    }
    (void)W;
    // Work items: one warp per (32 columns x kRows rows) tile; a tile whose source rows cost more
    // than a fair share is split along the source rows into partial items, longest first.
    p->H = std::max(B.Amax, 1);
    int rc;
    if ((rc = upload(p, &p->d_rows, p->h_rows.data(), p->h_rows.size())) != CGEF_OK) return rc;
    if (on_device) {
      if ((rc = device_band_tables(p, dr.sdp, dr.cc, dr.area, dr.sdl, dr.nweights, dr.host_rows)) != CGEF_OK)
        return rc;
    } else {
      const double no_weights = 0.0;  // a footprint without entries still gets a one-element table
      if ((rc = upload(p, &p->d_w, p->h_whalf.empty() ? &no_weights : p->h_whalf.data(),
                       std::max<size_t>(p->h_whalf.size(), 1))) != CGEF_OK)
        return rc;
      if ((rc = upload(p, &p->d_den_zf, den_zf.data(), den_zf.size())) != CGEF_OK) return rc;
    }
    const unsigned long long queue0[2] = {0, 0};
    if ((rc = upload(p, &p->d_queue, queue0, 2)) != CGEF_OK) return rc;
    if ((rc = rebuild_schedule(p, CGEF_SPLIT_WAVES, 0)) != CGEF_OK) return rc;
    // Mirrored columns may be paired when every row's interval is symmetric, or when the only
    // asymmetric rows close a periodic ring (their +a column is their -a column).
    bool symmetric = true;
    for (const BandRow& r : p->h_rows)
      if (r.a >= 0 && r.hi != r.a) symmetric = false;
    p->paired = CGEF_PAIRED && (symmetric || p->periodic_x);
    if ((rc = build_row_spectra(p)) != CGEF_OK) return rc;
  } else if (p->engine == CGEF_ENGINE_SEPARABLE) {
    // Filtering.jl:1391-1463: square truncation, lim = ceil(rad / step), point-sampled profile.
    p->di_lim = p->dx > 0 ? static_cast<int>(std::ceil(p->rad / p->dx)) : 0;
    p->sep_dj_lim = p->dy > 0 ? static_cast<int>(std::ceil(p->rad / p->dy)) : 0;
    p->dj_lim = p->sep_dj_lim;
    p->di_max = p->di_lim;
    for (int k = -p->di_lim; k <= p->di_lim; ++k)
      gx.push_back(kernel_weight(CGEF_GAUSSIAN, p->alpha, std::fabs(static_cast<double>(k) * p->dx), p->scale));
    for (int k = -p->sep_dj_lim; k <= p->sep_dj_lim; ++k)
      gy.push_back(kernel_weight(CGEF_GAUSSIAN, p->alpha, std::fabs(static_cast<double>(k) * p->dy), p->scale));
    auto profile = [](int lim, const std::vector<double>& g, int n, int periodic) {
      std::vector<double> out(n);
      for (int i = 0; i < n; ++i) {
        double s = 0.0;
        for (int dd = -lim; dd <= lim; ++dd) {
          int ii = i + dd;
          if ((ii >= 0 && ii < n) || periodic) s += g[dd + lim];
        }
        out[i] = s;
      }
      return out;
    };
    px = profile(p->di_lim, gx, nx, p->periodic_x);
    py = profile(p->sep_dj_lim, gy, ny, p->periodic_y);
    p->H = std::max(p->di_lim, 1);
    int rc;
    if ((rc = upload(p, &p->d_gx, gx.data(), gx.size())) != CGEF_OK) return rc;
    if ((rc = upload(p, &p->d_gy, gy.data(), gy.size())) != CGEF_OK) return rc;
    if ((rc = upload(p, &p->d_px, px.data(), px.size())) != CGEF_OK) return rc;
    if ((rc = upload(p, &p->d_py, py.data(), py.size())) != CGEF_OK) return rc;
  } else if (p->engine == CGEF_ENGINE_SPECTRAL) {
    // FFTWExt.jl:121-181: the transforms and the transfer function on the rfft grid
    p->H = 1;
    if (int rc = build_spectral(p)) return rc;
  } else {
    // Prefix-sum top-hat (Filtering.jl:833-907): measure factors, the tripled periodic axis,
    // the row band and per (row, band slot) the support half-width (Filtering.jl:990-1005).
    const double wxv = p->dx;
    p->x_period = (p->periodic_x && nx > 1) ? nx * p->dx : 0.0;
    p->y_period = (p->periodic_y && ny > 1) ? ny * p->dy : 0.0;
    const double dy_phys = sphere ? p->R * p->dy : p->dy;
    int lim = (std::isfinite(dy_phys) && dy_phys > 0) ? static_cast<int>(std::ceil(p->rad / dy_phys)) : 0;
    p->dj_lim = std::min(lim, ny - 1);
    p->pre_nrep = (p->periodic_x && nx > 1) ? 3 : 1;
    p->pre_ne = p->pre_nrep * nx;
    xe.resize(p->pre_ne);
    for (int r = 0; r < p->pre_nrep; ++r)
      for (int t = 0; t < nx; ++t)
        xe[static_cast<size_t>(r) * nx + t] =
            p->h_x[t] + (p->pre_nrep == 3 ? static_cast<double>(r - 1) * p->x_period : 0.0);
    prefix_wx.resize(p->pre_ne + 1);
    prefix_wx[0] = 0.0;
    for (int k = 0; k < p->pre_ne; ++k) prefix_wx[k + 1] = prefix_wx[k] + wxv;
    const int nbs = std::min(2 * p->dj_lim + 1, ny);
    p->pre_nb = nbs;
    prows.assign(static_cast<size_t>(ny) * nbs, PrefixRow{-1, 0, 0, 0, 0.0, 0.0});
    const bool uniform_fast = !p->periodic_x && p->pre_ne == nx && p->dx > 0;
    for (int j = 0; j < ny; ++j) {
      const double y_t = p->h_y[j];
      for (int b = 0; b < nbs; ++b) {
        PrefixRow& pr = prows[static_cast<size_t>(j) * nbs + b];
        int jj_raw = j - p->dj_lim + b;
        if (!(p->periodic_y || (jj_raw >= 0 && jj_raw < ny))) continue;
        int jj = ((jj_raw % ny) + ny) % ny;
        double dyv = p->h_y[jj] - y_t;
        if (p->periodic_y && p->y_period > 0.0) dyv -= p->y_period * std::round(dyv / p->y_period);
        double hw = metric_band(p->geometry, p->R, y_t, y_t + dyv, p->rad);
        if (hw < 0.0) continue;
        pr.jj = jj;
        pr.hw = hw;
        pr.wy = sphere ? p->R * p->R * std::cos(p->h_y[jj]) * p->dy : p->dy;
        if (p->periodic_x && p->pre_ne > nx && 2.0 * hw >= p->x_period) {
          pr.mode = 1;
        } else if (uniform_fast) {
          int w = 0;
          while ((w + 1) * p->dx <= hw) ++w;
          pr.mode = 2;
          pr.w = w;
        } else {
          pr.mode = 3;
        }
      }
    }
    p->H = 1;
    int rc;
    if ((rc = upload(p, &p->d_xe, xe.data(), xe.size())) != CGEF_OK) return rc;
    if ((rc = upload(p, &p->d_prefix_wx, prefix_wx.data(), prefix_wx.size())) != CGEF_OK) return rc;
    if ((rc = upload(p, &p->d_prows, prows.data(), prows.size())) != CGEF_OK) return rc;
  }

  int rc;
  if ((rc = upload(p, &p->d_x, p->h_x.data(), nx)) != CGEF_OK) return rc;
  if ((rc = upload(p, &p->d_sinlam, sinlam.data(), nx)) != CGEF_OK) return rc;
  if ((rc = upload(p, &p->d_coslam, coslam.data(), nx)) != CGEF_OK) return rc;
  if ((rc = upload(p, &p->d_sinphi, sinphi.data(), ny)) != CGEF_OK) return rc;
  if ((rc = upload(p, &p->d_cosphi, cosphi.data(), ny)) != CGEF_OK) return rc;
  if ((rc = upload(p, &p->d_area, area.data(), ny)) != CGEF_OK) return rc;
  if ((rc = upload(p, &p->d_xscale, xscale.data(), ny)) != CGEF_OK) return rc;
  if ((rc = upload(p, &p->d_tanfac, tanfac.data(), ny)) != CGEF_OK) return rc;
  if (!p->h_mask.empty())
    if ((rc = upload(p, &p->d_mask, p->h_mask.data(), p->h_mask.size())) != CGEF_OK) return rc;
  return CGEF_OK;
}

}  // namespace cgef
