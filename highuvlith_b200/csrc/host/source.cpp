// Pupil fills, scalar pupils and adaptive source sampling (FP64, host).
//
// Fills follow crates/highuvlith-core/src/source.rs:1178-1248; pupils follow
// optics/mod.rs:155-171,310-357 and optics/euv.rs:129-160; the sampler follows
// the algorithm of aerial.rs:357-947 (probe + zoom, rotated lattice laid out
// in the fundamental domain of the sampling box and mirrored, cells integrated
// on 8x8 sub-samples at hard edges, graded cells refined).  The constants
// that define that algorithm (probe sizes, thresholds, lattice rotation) have
// to be the same values for the point sets, and hence the kernels, to agree.
#include <algorithm>
#include <cmath>
#include <limits>

#include "host.hpp"

namespace huv {

namespace {
constexpr double kPi = 3.14159265358979323846;
constexpr double kProbeHalf = 2.0;
constexpr int kProbePoints = 129;
constexpr int kZoomPoints = 129;
constexpr int kMaxZoom = 6;
constexpr double kSupportThreshold = 1e-4;
constexpr double kResolvedCells = 24.0;
constexpr double kTargetStep = 0.04;
constexpr double kMinPoints = 200.0;
constexpr int kSub = 8;
constexpr int kMaxRefine = 8;
constexpr int kMaxRefineDepth = 3;
// cos/sin of the lattice rotation atan(1/golden ratio).
constexpr double kLatCos = 0.85065080835204;
constexpr double kLatSin = 0.5257311121191336;
constexpr int kMaxPerAxis = 128;
constexpr double kCoherentExtent = 1e-3;

inline double clean(double v) { return (std::isfinite(v) && v > 0.0) ? v : 0.0; }
inline double round_half_away(double x) { return std::round(x); }
}  // namespace

// ------------------------------------------------------------------ fills
void Fill::prepare() {
  if (kind == HUV_FILL_DIPOLE) {
    const double orient = p[2] * (kPi / 180.0);
    const double poles[2] = {orient, orient + kPi};
    for (int i = 0; i < 2; ++i) {
      pole[i][0] = p[0] * std::cos(poles[i]);
      pole[i][1] = p[0] * std::sin(poles[i]);
    }
  }
}

static double wrap_deg(double d) {
  // ((d + 180) rem_euclid 360) - 180
  double r = std::fmod(d + 180.0, 360.0);
  if (r < 0) r += 360.0;
  return r - 180.0;
}

double Fill::operator()(double x, double y) const {
  switch (kind) {
    case HUV_FILL_CONVENTIONAL: {
      const double rho = std::sqrt(x * x + y * y);
      return rho <= p[0] ? 1.0 : 0.0;
    }
    case HUV_FILL_ANNULAR: {
      const double rho = std::sqrt(x * x + y * y);
      return (rho >= p[0] && rho <= p[1]) ? 1.0 : 0.0;
    }
    case HUV_FILL_QUADRUPOLE: {
      const double angle = std::atan2(y, x) * (180.0 / kPi);
      const double half_open = p[2] / 2.0;
      const double centres[4] = {0.0, 90.0, 180.0, 270.0};
      for (double c : centres) {
        const double da = wrap_deg(angle - c);
        const double cx = p[0] * std::cos(c * (kPi / 180.0));
        const double cy = p[0] * std::sin(c * (kPi / 180.0));
        const double dist = std::sqrt((x - cx) * (x - cx) + (y - cy) * (y - cy));
        if (std::fabs(da) <= half_open && dist <= p[1]) return 1.0;
      }
      return 0.0;
    }
    case HUV_FILL_DIPOLE: {
      for (int i = 0; i < 2; ++i) {
        const double dx = x - pole[i][0], dy = y - pole[i][1];
        if (std::sqrt(dx * dx + dy * dy) <= p[1]) return 1.0;
      }
      return 0.0;
    }
    case HUV_FILL_GAUSSIAN: {
      const double rho = std::sqrt(x * x + y * y);
      if (rho <= 1.0 && p[0] > 0.0) return std::exp(-rho * rho / (2.0 * p[0] * p[0]));
      return 0.0;
    }
    case HUV_FILL_QUASAR: {
      const double rho = std::sqrt(x * x + y * y);
      if (rho < p[0] || rho > p[1]) return 0.0;
      const double angle = std::atan2(y, x) * (180.0 / kPi);
      const double half_open = p[2] / 2.0;
      const double centres[4] = {45.0, 135.0, 225.0, 315.0};
      for (double c : centres)
        if (std::fabs(wrap_deg(angle - c)) <= half_open) return 1.0;
      return 0.0;
    }
    default:
      return 0.0;
  }
}

// ------------------------------------------------------------------ optics
double defocus_phase(double z, double na_rho, double medium, double lambda, bool paraxial) {
  const double s = na_rho / medium;
  const double s2 = s * s;
  if (paraxial) return kPi * z * medium * s2 / lambda;
  const double c = std::sqrt(std::max(1.0 - s2, 0.0));
  return 2.0 * kPi * medium * z * s2 / ((1.0 + c) * lambda);
}

cd Optics::pupil(double fx, double fy, double z, double lambda) const {
  const double rho2 = fx * fx + fy * fy;
  if (rho2 > 1.0) return cd(0, 0);
  const double rho = std::sqrt(rho2);
  if (kind == HUV_OPTICS_EUV) {
    if (rho < obscuration) return cd(0, 0);
    const double ph = (z == 0.0) ? 0.0 : defocus_phase(z, na * rho, 1.0, lambda, paraxial);
    const double amp = std::sqrt(std::max(transmission, 0.0));
    return cd(amp * std::cos(ph), amp * std::sin(ph));
  }
  const double ph = (z == 0.0) ? 0.0 : defocus_phase(z, na * rho, medium, lambda, paraxial);
  return cd(std::cos(ph), std::sin(ph));
}

// ------------------------------------------------------------------ sampler
namespace {

struct Probe {
  double bx0, bx1, by0, by1, step_x, step_y;
  long count;
  double cx, cy;
};

bool probe_lattice(const Fill& f, double x0, double x1, double y0, double y1, int n, bool centered,
                   Probe& out) {
  const double step_x = (x1 - x0) / (n - 1);
  const double step_y = (y1 - y0) / (n - 1);
  const double half = (n - 1) / 2.0;
  std::vector<double> xs(n), ys(n);
  for (int i = 0; i < n; ++i) {
    xs[i] = centered ? (i - half) * step_x : x0 + i * step_x;
    ys[i] = centered ? (i - half) * step_y : y0 + i * step_y;
  }
  std::vector<double> vals(static_cast<size_t>(n) * n);
  double imax = 0.0;
  for (int iy = 0; iy < n; ++iy)
    for (int ix = 0; ix < n; ++ix) {
      const double v = clean(f(xs[ix], ys[iy]));
      vals[static_cast<size_t>(iy) * n + ix] = v;
      imax = std::max(imax, v);
    }
  if (imax <= 0.0) return false;
  const double thr = kSupportThreshold * imax;
  Probe p{std::numeric_limits<double>::max(), std::numeric_limits<double>::lowest(),
          std::numeric_limits<double>::max(), std::numeric_limits<double>::lowest(),
          step_x, step_y, 0, 0, 0};
  double wsum = 0, wx = 0, wy = 0;
  for (int iy = 0; iy < n; ++iy)
    for (int ix = 0; ix < n; ++ix) {
      const double v = vals[static_cast<size_t>(iy) * n + ix];
      if (v <= 0.0) continue;
      const double x = xs[ix], y = ys[iy];
      wsum += v;
      wx += v * x;
      wy += v * y;
      if (v > thr) {
        ++p.count;
        p.bx0 = std::min(p.bx0, x);
        p.bx1 = std::max(p.bx1, x);
        p.by0 = std::min(p.by0, y);
        p.by1 = std::max(p.by1, y);
      }
    }
  p.cx = wx / wsum;
  p.cy = wy / wsum;
  out = p;
  return true;
}

// Element of the sampling box's mirror group: (x, y) -> (+-a, +-b), (a, b) =
// (y, x) when swapped.
struct Mirror {
  bool swap, fx, fy;
  bool operator==(const Mirror& o) const { return swap == o.swap && fx == o.fx && fy == o.fy; }
  void apply(double x, double y, double& ox, double& oy) const {
    const double a = swap ? y : x, b = swap ? x : y;
    ox = fx ? -a : a;
    oy = fy ? -b : b;
  }
  Mirror then(const Mirror& h) const {  // self o h (apply h first)
    const bool hx = swap ? h.fy : h.fx;
    const bool hy = swap ? h.fx : h.fy;
    return Mirror{static_cast<bool>(swap ^ h.swap), static_cast<bool>(fx ^ hx), static_cast<bool>(fy ^ hy)};
  }
};

enum WallKind { WALL_X, WALL_Y, WALL_DIAG };

struct Cell {
  SourcePoint pt;
  bool graded;
  Mirror image;
};

struct Geometry {
  const Fill* f;
  double cx, cy, step, hx, hy;
  std::vector<WallKind> walls;

  void to_xy(double u, double v, double& x, double& y) const {
    x = step * (kLatCos * u - kLatSin * v);
    y = step * (kLatSin * u + kLatCos * v);
  }
  bool in_domain(double x, double y) const {
    if (!(std::fabs(x) <= hx && std::fabs(y) <= hy)) return false;
    for (WallKind w : walls) {
      if (w == WALL_X && !(x > 0.0)) return false;
      if (w == WALL_Y && !(y > 0.0)) return false;
      if (w == WALL_DIAG && !(y < x)) return false;
    }
    return true;
  }
  double eval(const Mirror& g, double x, double y) const {
    double gx, gy;
    g.apply(x, y, gx, gy);
    return clean((*f)(cx + gx, cy + gy));
  }
  SourcePoint point(const Mirror& g, double x, double y, double w) const {
    double gx, gy;
    g.apply(x, y, gx, gy);
    return SourcePoint{cx + gx, cy + gy, w};
  }

  bool integrate(double u0, double v0, double du, const Mirror& g, Cell& out) const {
    const double area = du * du;
    double ccx, ccy;
    to_xy(u0 + 0.5 * du, v0 + 0.5 * du, ccx, ccy);
    const double corner_uv[4][2] = {{0.0, 0.0}, {du, 0.0}, {0.0, du}, {du, du}};
    double kx[4], ky[4];
    bool interior = true;
    for (int c = 0; c < 4; ++c) {
      to_xy(u0 + corner_uv[c][0], v0 + corner_uv[c][1], kx[c], ky[c]);
      interior = interior && in_domain(kx[c], ky[c]);
    }
    const double vc = eval(g, ccx, ccy);
    if (interior) {
      bool uniform = true;
      for (int c = 0; c < 4 && uniform; ++c) uniform = eval(g, kx[c], ky[c]) == vc;
      if (uniform) {
        if (!(vc > 0.0)) return false;
        out = Cell{point(g, ccx, ccy, vc * area), false, g};
        return true;
      }
    }
    const double sub = static_cast<double>(kSub);
    double mass = 0, mx = 0, my = 0, vmin = std::numeric_limits<double>::infinity(), vmax = 0;
    int inside = 0, lit = 0;
    for (int k = 0; k < kSub * kSub; ++k) {
      const double a = static_cast<double>(k % kSub), b = static_cast<double>(k / kSub);
      double x, y;
      to_xy(u0 + (a + 0.5) / sub * du, v0 + (b + 0.5) / sub * du, x, y);
      if (!in_domain(x, y)) continue;
      ++inside;
      const double v = eval(g, x, y);
      vmin = std::min(vmin, v);
      vmax = std::max(vmax, v);
      if (v > 0.0) {
        mass += v;
        mx += v * x;
        my += v * y;
        ++lit;
      }
    }
    if (!(mass > 0.0)) return false;
    const bool graded = lit == inside && vmin < vmax;
    if (interior && lit == kSub * kSub && vc > 0.0)
      out = Cell{point(g, ccx, ccy, vc * area), graded, g};
    else
      out = Cell{point(g, mx / mass, my / mass, mass / (sub * sub) * area), graded, g};
    return true;
  }

  void refine(double u0, double v0, double du, const Cell& cell, double target, int depth,
              std::vector<SourcePoint>& out) const {
    if (!(cell.graded && cell.pt.w > target) || depth >= kMaxRefineDepth) {
      out.push_back(cell.pt);
      return;
    }
    int r = static_cast<int>(std::ceil(std::sqrt(cell.pt.w / target)));
    r = std::min(std::max(r, 2), kMaxRefine);
    const double dc = du / r;
    for (int b = 0; b < r; ++b)
      for (int a = 0; a < r; ++a) {
        const double cu = u0 + a * dc, cv = v0 + b * dc;
        Cell child;
        if (integrate(cu, cv, dc, cell.image, child)) refine(cu, cv, dc, child, target, depth + 1, out);
      }
  }
};

std::vector<Mirror> mirror_group(const std::vector<Mirror>& gens) {
  std::vector<Mirror> group{Mirror{false, false, false}};
  for (size_t k = 0; k < group.size(); ++k)
    for (const Mirror& g : gens) {
      const Mirror e = group[k].then(g);
      if (std::find(group.begin(), group.end(), e) == group.end()) group.push_back(e);
    }
  return group;
}

std::vector<SourcePoint> lattice_cells(const Fill& f, double cx, double cy, double w, double h,
                                       double step, bool sx, bool sy, bool diag) {
  Geometry geo{&f, cx, cy, step, 0.5 * w, 0.5 * h, {}};
  std::vector<Mirror> gens;
  if (sx && !diag) {
    geo.walls.push_back(WALL_X);
    gens.push_back(Mirror{false, true, false});
  }
  if (sy) {
    geo.walls.push_back(WALL_Y);
    gens.push_back(Mirror{false, false, true});
  }
  if (diag) {
    geo.walls.push_back(WALL_DIAG);
    gens.push_back(Mirror{true, false, false});
  }
  const double margin = step * std::sqrt(2.0);
  const double reach = std::hypot(w, h) * 0.5 + margin;
  const long n = static_cast<long>(std::ceil(reach / step)) + 1;
  std::vector<std::pair<double, double>> cells;
  for (long j = -n; j < n; ++j)
    for (long i = -n; i < n; ++i) {
      double x, y;
      geo.to_xy(i + 0.5, j + 0.5, x, y);
      const bool near_domain = (!sx || diag || x > -margin) && (!sy || y > -margin) &&
                               (!diag || y < x + margin);
      const bool near_box = std::fabs(x) <= 0.5 * w + margin && std::fabs(y) <= 0.5 * h + margin;
      if (near_box && near_domain) cells.emplace_back(static_cast<double>(i), static_cast<double>(j));
    }
  const std::vector<Mirror> group = mirror_group(gens);
  const size_t n_img = group.size();
  const size_t total_cells = cells.size() * n_img;
  std::vector<Cell> coarse(total_cells);
  std::vector<char> ok(total_cells, 0);
  parallel_for(static_cast<int64_t>(total_cells), [&](int64_t b, int64_t e) {
    for (int64_t k = b; k < e; ++k) {
      const auto& c = cells[k / n_img];
      ok[k] = geo.integrate(c.first, c.second, 1.0, group[k % n_img], coarse[k]) ? 1 : 0;
    }
  });
  double total = 0.0;
  for (size_t k = 0; k < total_cells; ++k)
    if (ok[k]) total += coarse[k].pt.w;
  const double target = total / kMinPoints;
  std::vector<SourcePoint> out;
  for (size_t k = 0; k < total_cells; ++k) {
    if (!ok[k]) continue;
    const auto& c = cells[k / n_img];
    geo.refine(c.first, c.second, 1.0, coarse[k], target, 0, out);
  }
  return out;
}

std::vector<SourcePoint> normalized_or_centroid(std::vector<SourcePoint> pts, double cx, double cy) {
  double total = 0.0;
  for (const auto& p : pts) total += p.w;
  if (pts.empty() || std::isnan(total) || total <= 0.0) return {SourcePoint{cx, cy, 1.0}};
  for (auto& p : pts) p.w /= total;
  return pts;
}

}  // namespace

std::vector<SourcePoint> sample_source(const Fill& f, int points_per_axis, double df_sigma) {
  Probe probe;
  if (!probe_lattice(f, -kProbeHalf, kProbeHalf, -kProbeHalf, kProbeHalf, kProbePoints, true, probe))
    throw Error(HUV_ERR_INVALID_PARAMETER,
                "illumination: source pupil fill has no intensity inside |sigma| <= 2");
  for (int level = 0; level < kMaxZoom; ++level) {
    const bool rx = probe.bx1 - probe.bx0 >= kResolvedCells * probe.step_x;
    const bool ry = probe.by1 - probe.by0 >= kResolvedCells * probe.step_y;
    if (rx && ry) break;
    Probe p;
    if (!probe_lattice(f, probe.bx0 - probe.step_x, probe.bx1 + probe.step_x, probe.by0 - probe.step_y,
                       probe.by1 + probe.step_y, kZoomPoints, false, p))
      break;
    probe = p;
  }
  const bool sym_x = std::fabs(probe.bx0 + probe.bx1) <= 0.5 * probe.step_x;
  const bool sym_y = std::fabs(probe.by0 + probe.by1) <= 0.5 * probe.step_y;
  double cx_box, w, cy_box, h;
  if (sym_x) {
    cx_box = 0.0;
    w = 2.0 * (std::max(std::fabs(probe.bx0), std::fabs(probe.bx1)) + probe.step_x);
  } else {
    cx_box = 0.5 * (probe.bx0 + probe.bx1);
    w = probe.bx1 - probe.bx0 + 2.0 * probe.step_x;
  }
  if (sym_y) {
    cy_box = 0.0;
    h = 2.0 * (std::max(std::fabs(probe.by0), std::fabs(probe.by1)) + probe.step_y);
  } else {
    cy_box = 0.5 * (probe.by0 + probe.by1);
    h = probe.by1 - probe.by0 + 2.0 * probe.step_y;
  }
  if (sym_x && sym_y && std::fabs(w - h) <= std::max(probe.step_x, probe.step_y)) {
    const double m = std::max(w, h);
    w = h = m;
  }
  const double extent = std::max(w, h);
  if (points_per_axis == 1 || extent < kCoherentExtent * df_sigma)
    return {SourcePoint{sym_x ? 0.0 : probe.cx, sym_y ? 0.0 : probe.cy, 1.0}};
  if (points_per_axis > 0) {
    const double step = extent / points_per_axis;
    const int nx = std::max(static_cast<int>(round_half_away(w / step)), 1);
    const int ny = std::max(static_cast<int>(round_half_away(h / step)), 1);
    const double hx = w / nx, hy = h / ny;
    std::vector<SourcePoint> pts;
    for (int iy = 0; iy < ny; ++iy) {
      const double y = cy_box + (iy + 0.5 - ny / 2.0) * hy;
      for (int ix = 0; ix < nx; ++ix) {
        const double x = cx_box + (ix + 0.5 - nx / 2.0) * hx;
        const double v = f(x, y);
        if (std::isfinite(v) && v > 0.0) pts.push_back(SourcePoint{x, y, v});
      }
    }
    return normalized_or_centroid(std::move(pts), probe.cx, probe.cy);
  }
  const double area = static_cast<double>(std::max(probe.count, 1L)) * probe.step_x * probe.step_y;
  const double step =
      std::max(std::min(kTargetStep, std::sqrt(area / kMinPoints)), extent / kMaxPerAxis);
  const bool diag = sym_x && sym_y && w == h;
  return normalized_or_centroid(lattice_cells(f, cx_box, cy_box, w, h, step, sym_x, sym_y, diag),
                                probe.cx, probe.cy);
}

}  // namespace huv
