/*
 * trk_aperture.cpp -- the line-mode dynamic-aperture search of elegant
 * (do_aperture_search_line, src/aperture_search.c:985-1234, with the area of
 * trimApertureSearchResult, src/trimApertureSearchResult.c) as a driver of
 * the batched tracking launch.
 *
 * The reference tracks one particle at a time along each line and stops a
 * sweep at the first loss.  Particles do not interact on this path, so every
 * point of a sweep, of every line and of every error seed is tracked in one
 * launch (trk_track for one lattice, trk_track_ensemble for several) and the
 * first loss along each line is read afterwards: the same survivor and loss
 * points as the serial search.  Each refinement sweep (split) depends on the
 * previous one, so a search takes 1 + n_splits launches.
 */
#include <cmath>
#include <cstring>
#include <vector>

#include "trk.h"
#include "trk_lattice.h"

namespace {

/* line directions (src/aperture_search.c:1016-1045) */
void line_factors(int lines, int full_plane, std::vector<double> &dxf, std::vector<double> &dyf) {
  dxf.assign(lines, 0.0);
  dyf.assign(lines, 0.0);
  const double PI = 3.141592653589793238462643;
  switch (lines) {
  case 1:
    dxf[0] = 1;
    dyf[0] = 1;
    break;
  case 2:
    dxf[0] = -1;
    dyf[0] = 1;
    dxf[1] = 1;
    dyf[1] = 1;
    break;
  case 3:
    dxf[0] = 0;
    dyf[0] = 1;
    dxf[1] = dyf[1] = 1 / std::sqrt(2.0);
    dxf[2] = 1;
    dyf[2] = 0;
    break;
  default: {
    const double dtheta = full_plane == 0 ? PI / (lines - 1) : 2 * PI / (lines - 1);
    for (int l = 0; l < lines; l++) {
      dxf[l] = std::sin(-PI / 2 + dtheta * l);
      dyf[l] = std::cos(-PI / 2 + dtheta * l);
      if (std::fabs(dxf[l]) < 1e-6)
        dxf[l] = 0;
      if (std::fabs(dyf[l]) < 1e-6)
        dyf[l] = 0;
    }
  }
  }
}

/* one pass of the island clipping and the trapezoid area
 * (trimApertureSearchResult1, src/trimApertureSearchResult.c:16-104) */
double trim_once(int lines, double *x, double *y, const double *dxf, const double *dyf, int full_plane) {
  if (!full_plane) {
    for (int l = 0; l < lines / 2; l++)
      if (x[l + 1] < x[l])
        x[l + 1] = x[l];
    for (int l = lines - 1; l > lines / 2; l--)
      if (x[l - 1] > x[l])
        x[l - 1] = x[l];
    for (int l = lines / 2; l > 0; l--)
      if (y[l - 1] > y[l])
        y[l - 1] = y[l];
    for (int l = lines / 2; l < lines - 1; l++)
      if (y[l + 1] > y[l])
        y[l + 1] = y[l];
  } else {
    for (int l = 0; l < lines - 1; l++) {
      if (dxf[l] > 0 && dxf[l + 1] > 0) {
        if (dyf[l] > 0 && dyf[l + 1] > 0) {
          if (x[l + 1] < x[l])
            x[l] = x[l + 1];
        } else if (dyf[l] < 0 && dyf[l + 1] < 0) {
          if (x[l + 1] > x[l])
            x[l + 1] = x[l];
        }
      } else if (dxf[l] < 0 && dxf[l + 1] < 0) {
        if (dyf[l] > 0 && dyf[l + 1] > 0) {
          if (x[l + 1] < x[l])
            x[l + 1] = x[l];
        } else if (dyf[l] < 0 && dyf[l + 1] < 0) {
          if (x[l + 1] > x[l])
            x[l] = x[l + 1];
        }
      }
    }
    for (int l = 0; l < lines - 1; l++) {
      if (dxf[l] > 0 && dxf[l + 1] > 0) {
        if (dyf[l] > 0 && dyf[l + 1] > 0) {
          if (y[l + 1] > y[l])
            y[l + 1] = y[l];
        } else if (dyf[l] < 0 && dyf[l + 1] < 0) {
          if (y[l] < y[l + 1])
            y[l] = y[l + 1];
        }
      } else if (dxf[l] < 0 && dxf[l + 1] < 0) {
        if (dyf[l] > 0 && dyf[l + 1] > 0) {
          if (y[l + 1] < y[l])
            y[l] = y[l + 1];
        } else if (dyf[l] < 0 && dyf[l + 1] < 0) {
          if (y[l + 1] < y[l])
            y[l + 1] = y[l];
        }
      }
    }
  }
  double area = 0;
  for (int l = 0; l < lines - 1; l++)
    area += (x[l + 1] - x[l]) * (y[l + 1] + y[l]) / 2;
  return area;
}

/* trimApertureSearchResult: repeat until the area stops changing, at most
 * `lines` times */
double trim(int lines, double *x, double *y, const double *dxf, const double *dyf, int full_plane) {
  double area1 = -1, area2 = -1;
  long count = lines;
  while (count-- && (area2 = trim_once(lines, x, y, dxf, dyf, full_plane)) != area1)
    area1 = area2;
  return area1;
}

/* the search state of one line of one variant */
struct Line {
  double x0, y0, dx, dy;
  long steps;
  double xs, ys;            /* survived */
  double xl, yl, sl;        /* lost */
};

} // namespace

extern "C" int trk_aperture_search_lines(trk_context *ctx, const trk_lattice *const *lattices, int n_variants,
                                         const trk_aperture_search *search, const trk_run *run, double *x_limit,
                                         double *y_limit, double *x_clipped, double *y_clipped, double *x_lost,
                                         double *y_lost, double *s_lost, double *area) {
  if (!ctx || !lattices || !search || !run || n_variants < 1 || !x_limit || !y_limit)
    return trk_set_error(TRK_ERR_ARG, "null argument");
  const trk_aperture_search &S = *search;
  const int L = S.lines;
  if (L < 1)
    return trk_set_error(TRK_ERR_ARG, "at least one line");
  if (S.nx < 2)
    return trk_set_error(TRK_ERR_ARG, "nx must be at least 2");
  if (S.n_splits < 0 || (S.n_splits > 0 && !(S.split_fraction > 0 && S.split_fraction < 1)))
    return trk_set_error(TRK_ERR_ARG, "split_fraction must be in (0, 1)");
  for (int v = 0; v < n_variants; v++)
    if (!lattices[v])
      return trk_set_error(TRK_ERR_ARG, "null lattice %d", v);
  std::vector<double> dxf, dyf;
  line_factors(L, S.full_plane, dxf, dyf);

  std::vector<Line> st((size_t)n_variants * L);
  for (int v = 0; v < n_variants; v++)
    for (int l = 0; l < L; l++) {
      Line &q = st[(size_t)v * L + l];
      if (dxf[l] > 0)
        q.xs = q.ys = -1;
      else
        q.xs = -(q.ys = -1);
      q.xl = q.yl = q.sl = 1.7976931348623157e308;
      const double ex = S.slope_mode ? S.xpmax : S.xmax, ey = S.slope_mode ? S.ypmax : S.ymax;
      q.dx = ex / (S.nx - 1) * dxf[l];
      q.dy = ey / (S.nx - 1) * dyf[l];
      q.x0 = q.y0 = 0;
      q.steps = S.nx;
    }
  /* origin (index 0 of the first sweep) of each variant: whether it survived */
  std::vector<char> origin_stable(n_variants, 0);

  std::vector<double> rows, out;
  std::vector<long> lost_pass;
  std::vector<long> offsets(n_variants + 1);
  int rc;
  for (int split = 0; split <= S.n_splits; split++) {
    if (split > 0)
      for (Line &q : st) {
        q.x0 = q.xs;
        q.y0 = q.ys;
        q.dx *= S.split_fraction;
        q.dy *= S.split_fraction;
        q.x0 += q.dx;
        q.y0 += q.dy;
        q.steps = (long)(1 / S.split_fraction - 0.5);
        if (q.steps < 1)
          q.steps = 1;
      }
    /* every point of every line of every variant, variant-major; id = row */
    long n = 0;
    for (int v = 0; v < n_variants; v++) {
      offsets[v] = n;
      for (int l = 0; l < L; l++)
        n += st[(size_t)v * L + l].steps;
    }
    offsets[n_variants] = n;
    rows.assign((size_t)n * 7, 0.0);
    long r = 0;
    for (int v = 0; v < n_variants; v++)
      for (int l = 0; l < L; l++) {
        const Line &q = st[(size_t)v * L + l];
        for (long k = 0; k < q.steps; k++, r++) {
          double *row = &rows[(size_t)r * 7];
          for (int c = 0; c < 6; c++)
            row[c] = S.orbit[c];
          if (!S.slope_mode) {
            row[0] = k * q.dx + q.x0 + S.orbit[0];
            row[2] = k * q.dy + q.y0 + S.orbit[2];
          } else {
            row[1] = k * q.dx + q.x0 + S.orbit[1];
            row[3] = k * q.dy + q.y0 + S.orbit[3];
          }
          row[6] = (double)(r + 1);
        }
      }
    if ((rc = trk_beam_load(ctx, rows.data(), n, 7)))
      return rc;
    trk_stats stats;
    if (n_variants == 1)
      rc = trk_track(ctx, lattices[0], run, &stats);
    else
      rc = trk_track_ensemble(ctx, lattices, n_variants, offsets.data(), run, &stats);
    if (rc)
      return rc;
    out.assign((size_t)n * 7, 0.0);
    lost_pass.assign(n, -1);
    long n_left = 0;
    if ((rc = trk_beam_store(ctx, out.data(), 7, &n_left, lost_pass.data(), nullptr)))
      return rc;
    /* rows come back survivors first: index them by id */
    std::vector<long> at(n, -1);
    for (long i = 0; i < n; i++) {
      const long id = (long)out[(size_t)i * 7 + 6] - 1;
      if (id >= 0 && id < n)
        at[id] = i;
    }
    r = 0;
    for (int v = 0; v < n_variants; v++)
      for (int l = 0; l < L; l++) {
        Line &q = st[(size_t)v * L + l];
        bool stopped = false;
        for (long k = 0; k < q.steps; k++, r++) {
          if (stopped)
            continue;
          const long i = at[r];
          const bool lost = i < 0 || lost_pass[i] >= 0;
          if (lost) {
            /* the sweep ends at the first loss (src/aperture_search.c:1135-1151) */
            if (i >= 0) {
              q.xl = out[(size_t)i * 7 + 0];
              q.yl = out[(size_t)i * 7 + 2];
              q.sl = out[(size_t)i * 7 + 4];
            }
            stopped = true;
            continue;
          }
          if (k == 0 && split == 0)
            origin_stable[v] = 1;
          const double xk = q.x0 + k * q.dx, yk = q.y0 + k * q.dy;
          if (dxf[l]) {
            if ((dxf[l] > 0 && q.xs < xk) || (dxf[l] < 0 && q.xs > xk)) {
              q.xs = xk;
              q.ys = yk;
            }
          } else if (q.ys < yk) {
            q.xs = xk;
            q.ys = yk;
          }
        }
      }
  }
  std::vector<double> xc(L), yc(L);
  for (int v = 0; v < n_variants; v++) {
    for (int l = 0; l < L; l++) {
      const Line &q = st[(size_t)v * L + l];
      x_limit[(size_t)v * L + l] = xc[l] = q.xs;
      y_limit[(size_t)v * L + l] = yc[l] = q.ys;
      if (x_lost)
        x_lost[(size_t)v * L + l] = q.xl;
      if (y_lost)
        y_lost[(size_t)v * L + l] = q.yl;
      if (s_lost)
        s_lost[(size_t)v * L + l] = q.sl;
    }
    double a = 0;
    if (origin_stable[v] && L > 1)
      a = trim(L, xc.data(), yc.data(), dxf.data(), dyf.data(), S.full_plane);
    if (area)
      area[v] = a;
    for (int l = 0; l < L; l++) {
      if (x_clipped)
        x_clipped[(size_t)v * L + l] = xc[l];
      if (y_clipped)
        y_clipped[(size_t)v * L + l] = yc[l];
    }
  }
  return TRK_OK;
}

/* do_aperture_search_grid (src/aperture_search.c:1236-1521) over n_variants
 * lattices: each side's grid for every variant in one launch, then the
 * reference's column reduction (survivors raise v_limit, a loss nearer the
 * origin lowers it again) and area. */
extern "C" int trk_aperture_search_grid(trk_context *ctx, const trk_lattice *const *lattices, int n_variants,
                                        const trk_aperture_grid *grid, const trk_run *run, double *u_limit,
                                        double *v_limit, double *x_lost, double *y_lost, double *s_lost,
                                        double *delta_lost, double *area) {
  if (!ctx || !lattices || !grid || !run || n_variants < 1 || !v_limit)
    return trk_set_error(TRK_ERR_ARG, "null argument");
  for (int v = 0; v < n_variants; v++)
    if (!lattices[v])
      return trk_set_error(TRK_ERR_ARG, "null lattice %d", v);
  const trk_aperture_grid &G = *grid;
  int icu, icv;
  long nu, nv;
  double umin, umax, vmin, vmax;
  if (G.delta_mode == 1) { /* DELTA_X_MODE */
    icu = 5, icv = 0, nu = G.ndelta, umin = G.deltamin, umax = G.deltamax, nv = G.nx, vmin = G.xmin, vmax = G.xmax;
  } else if (G.delta_mode == 2) { /* DELTA_Y_MODE */
    icu = 5, icv = 2, nu = G.ndelta, umin = G.deltamin, umax = G.deltamax, nv = G.ny, vmin = G.ymin, vmax = G.ymax;
  } else if (G.delta_mode == 0) {
    icu = 0, icv = 2, nu = G.nx, umin = G.xmin, umax = G.xmax, nv = G.ny, vmin = G.ymin, vmax = G.ymax;
  } else
    return trk_set_error(TRK_ERR_ARG, "delta_mode must be 0, 1 or 2");
  if (nu < 2 || nv < 2)
    return trk_set_error(TRK_ERR_ARG, "grid needs at least 2 points per axis");
  const double DMAX = 1.7976931348623157e308;
  const double du = (umax - umin) / (nu - 1);
  const int sides = vmin < 0 ? 2 : 1;
  const size_t per = (size_t)nu * nv;
  const long n = (long)(per * n_variants);
  for (int v = 0; v < n_variants; v++) {
    if (area)
      area[v] = 0;
    for (int side = 0; side < 2; side++)
      for (long iu = 0; iu < nu; iu++) {
        const size_t o = ((size_t)v * 2 + side) * nu + iu;
        v_limit[o] = 0;
        if (u_limit)
          u_limit[o] = 0;
        if (x_lost)
          x_lost[o] = DMAX;
        if (y_lost)
          y_lost[o] = DMAX;
        if (s_lost)
          s_lost[o] = DMAX;
        if (delta_lost)
          delta_lost[o] = DMAX;
      }
  }
  std::vector<double> rows((size_t)n * 7), out((size_t)n * 7);
  std::vector<long> lost_pass(n), offsets(n_variants + 1), at(n);
  std::vector<double> vl(nu), vl1(nu), xl(nu), yl(nu), sl(nu), dl(nu);
  for (int v = 0; v <= n_variants; v++)
    offsets[v] = (long)(per * v);
  int rc;
  for (int side = 0; side < sides; side++) {
    const double dv = side == 0 ? vmax / (nv - 1) : vmin / (nv - 1);
    long r = 0;
    for (int v = 0; v < n_variants; v++)
      for (long iu = 0; iu < nu; iu++)
        for (long iv = 0; iv < nv; iv++, r++) {
          double *row = &rows[(size_t)r * 7];
          for (int c = 0; c < 6; c++)
            row[c] = 0;
          row[icu] = iu * du + umin;
          row[icv] = iv * dv;
          for (int c = 0; c < 6; c++)
            row[c] += G.orbit[c];
          row[6] = (double)(r + 1);
        }
    if ((rc = trk_beam_load(ctx, rows.data(), n, 7)))
      return rc;
    trk_stats stats;
    rc = n_variants == 1 ? trk_track(ctx, lattices[0], run, &stats)
                         : trk_track_ensemble(ctx, lattices, n_variants, offsets.data(), run, &stats);
    if (rc)
      return rc;
    long n_left = 0;
    if ((rc = trk_beam_store(ctx, out.data(), 7, &n_left, lost_pass.data(), nullptr)))
      return rc;
    for (long i = 0; i < n; i++)
      at[i] = -1;
    for (long i = 0; i < n; i++) {
      const long id = (long)out[(size_t)i * 7 + 6] - 1;
      if (id >= 0 && id < n)
        at[id] = i;
    }
    for (int v = 0; v < n_variants; v++) {
      const long base = offsets[v];
      long survivors = 0;
      for (long iu = 0; iu < nu; iu++) {
        vl[iu] = 0;
        vl1[iu] = side == 0 ? vmax + dv : vmin + dv;
        xl[iu] = yl[iu] = sl[iu] = dl[iu] = DMAX;
      }
      /* survivors first, then the lost particles (src/aperture_search.c:1422-1449) */
      for (int pass = 0; pass < 2; pass++)
        for (long k = 0; k < (long)per; k++) {
          const long i = at[base + k];
          const bool lost = i < 0 || lost_pass[i] >= 0;
          if (lost != (pass == 1))
            continue;
          const long iu = k / nv, iv = k % nv;
          const double vv = iv * dv;
          if (!lost) {
            survivors++;
            if ((side == 0 && vv > vl[iu]) || (side == 1 && vv < vl[iu]))
              vl[iu] = vv;
            continue;
          }
          if ((side == 0 && vv < vl[iu]) || (side == 1 && vv > vl[iu]))
            vl[iu] = vv;
          if (i >= 0 && ((side == 0 && vv < vl1[iu]) || (side == 1 && vv > vl1[iu]))) {
            vl1[iu] = vv;
            xl[iu] = out[(size_t)i * 7 + 0];
            yl[iu] = out[(size_t)i * 7 + 2];
            sl[iu] = out[(size_t)i * 7 + 4];
            dl[iu] = out[(size_t)i * 7 + 5];
          }
        }
      double a = 0;
      if (survivors)
        for (long iu = 0; iu < nu; iu++)
          a += std::fabs(vl[iu] * du);
      if (area)
        area[v] += a;
      for (long iu = 0; iu < nu; iu++) {
        const size_t o = ((size_t)v * 2 + side) * nu + iu;
        v_limit[o] = vl[iu];
        if (u_limit)
          u_limit[o] = iu * du + umin;
        if (x_lost)
          x_lost[o] = xl[iu];
        if (y_lost)
          y_lost[o] = yl[iu];
        if (s_lost)
          s_lost[o] = sl[iu];
        if (delta_lost)
          delta_lost[o] = dl[iu];
      }
    }
  }
  return TRK_OK;
}
