/* Test infrastructure only: the CPU oracle (see fir_oracle.h).
 *
 * Each function restates one piece of FIR's algorithm in plain C, in FIR's
 * evaluation order and types (geometry in double, data in float, products of
 * a double length and a float value formed in double and rounded once on
 * accumulation), serially in FIR's loop order.  Built with
 * -ffp-contract=off so no multiply-add is fused.  Citations are paths inside
 * the FIR project.
 */
#include "fir_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define FO_EPS 0.00001          /* macros.h:8 */
#define FO_PI 3.141592653589793 /* macros.h:11 */

static double dmin(double a, double b) { return a < b ? a : b; } /* macros.h:4 */
static double dmax(double a, double b) { return a > b ? a : b; } /* macros.h:5 */

/* ---- projection geometry: ProjHeader.cc:6-106 (check), :108-186 (fill) ---- */
int fo_proj_fill(fo_proj* p)
{
  if (p->n_rings <= 0) return -1;
  if (p->n_crystals_per_ring <= 0 || p->n_crystals_per_ring % 4 != 0) return -2;
  if (p->segment_span <= 0 || p->segment_span % 2 != 1) return -3;
  const int max_span = 2 * p->n_rings - 1;
  if (p->segment_span > max_span) return -3;
  if (p->n_segments < 0 || p->n_segments % 2 != 1) return -4;
  int max_nseg = max_span / p->segment_span;
  max_nseg -= 1 - max_nseg % 2;
  if (p->n_segments > max_nseg) return -4;
  if (p->n_segments > FO_MAX_SEGMENTS) return -4;
  if (p->n_tang_coords < 0) return -5;
  if (p->n_tang_coords == 0)
    p->n_tang_coords = p->n_crystals_per_ring - 1;
  else if (p->n_tang_coords > p->n_crystals_per_ring - 1)
    return -5;

  p->seg_offset = (p->n_segments - 1) / 2;
  p->tang_offset = p->n_tang_coords / 2;
  for (int seg = -p->seg_offset; seg <= p->seg_offset; ++seg)
  {
    int len;
    const int a = abs(seg);
    if (p->segment_span == 1)
      len = p->n_rings - a;
    else
    {
      len = 2 * p->n_rings - 1;
      if (a >= 1) len -= p->segment_span + 1;
      if (a >= 2) len -= 2 * p->segment_span * (a - 1);
    }
    p->n_axial[seg + p->seg_offset] = len;
  }
  p->n_views = p->n_crystals_per_ring / 2;
  p->n_bins = 0;
  for (int i = 0; i < p->n_segments; ++i)
    p->n_bins += (long long)p->n_axial[i] * p->n_views * p->n_tang_coords;
  p->half_span = (p->segment_span - 1) / 2;
  if (p->segment_span == 1)
    p->max_ring_diff = p->seg_offset;
  else
  {
    p->max_ring_diff = p->half_span;
    if (p->seg_offset > 0) p->max_ring_diff += p->seg_offset * p->segment_span;
  }
  return 0;
}

/* ---- scanner: ScannerHeader.cc:26-303 (check), :305-342 (fill) ---- */
int fo_scanner_check(fo_scanner_params* s, int* n_rings, int* n_cpr)
{
  for (int i = 0; i < 3; ++i)
    if (s->crystal_dims[i] < 0 || s->module_dims[i] < 0 || s->rsector_dims[i] < 0) return -1;
  if (s->crystal_repeat[0] <= 0 || s->crystal_repeat[1] <= 0) return -1;
  if (s->module_repeat[0] <= 0 || s->module_repeat[1] <= 0) return -1;
  if (s->inter_crystal[0] < 0 || s->inter_crystal[1] < 0) return -1;
  if (s->inter_module[0] < 0 || s->inter_module[1] < 0) return -1;
  if (s->rsector_repeat <= 0 || s->rsector_inner_radius <= 0) return -1;
  if (s->crystal_repeat[0] > 1 && s->crystal_dims[1] == 0) return -1;
  if (s->crystal_repeat[1] > 1 && s->crystal_dims[2] == 0) return -1;

  const double min_mod[3] = {
    s->crystal_dims[0],
    s->crystal_dims[1] * s->crystal_repeat[0] + s->inter_crystal[0] * (s->crystal_repeat[0] - 1),
    s->crystal_dims[2] * s->crystal_repeat[1] + s->inter_crystal[1] * (s->crystal_repeat[1] - 1)};
  for (int i = 0; i < 3; ++i)
  {
    if (s->module_dims[i] == 0.0)
      s->module_dims[i] = min_mod[i];
    else if (s->module_dims[i] < min_mod[i])
      return -1;
  }
  if (s->module_repeat[0] > 1 && s->module_dims[1] == 0) return -1;
  if (s->module_repeat[1] > 1 && s->module_dims[2] == 0) return -1;
  const double min_rs[3] = {
    s->module_dims[0],
    s->module_dims[1] * s->module_repeat[0] + s->inter_module[0] * (s->module_repeat[0] - 1),
    s->module_dims[2] * s->module_repeat[1] + s->inter_module[1] * (s->module_repeat[1] - 1)};
  for (int i = 0; i < 3; ++i)
  {
    if (s->rsector_dims[i] == 0)
      s->rsector_dims[i] = min_rs[i];
    else if (s->rsector_dims[i] < min_rs[i])
      return -1;
  }
  if (n_cpr) *n_cpr = s->crystal_repeat[0] * s->module_repeat[0] * s->rsector_repeat;
  if (n_rings) *n_rings = s->crystal_repeat[1] * s->module_repeat[1];
  return 0;
}

/* ScannerData.cc:248-329 (crystal XY) and :331-377 (slice Z). */
int fo_scanner_tables(const fo_scanner_params* s0, double* xy, double* z)
{
  fo_scanner_params s = *s0;
  int n_rings, n_cpr;
  if (fo_scanner_check(&s, &n_rings, &n_cpr) != 0) return -1;

  const double cvy = s.crystal_dims[1] + s.inter_crystal[0];
  const double cvz = s.crystal_dims[2] + s.inter_crystal[1];
  const double mvy = s.module_dims[1] + s.inter_module[0];
  const double mvz = s.module_dims[2] + s.inter_module[1];
  const double tx = s.rsector_inner_radius + s.rsector_dims[0] / 2;
  const int crystal_offset = s.module_repeat[0] * s.crystal_repeat[0] / 2;

  const int ncy = s.crystal_repeat[0], nmy = s.module_repeat[0];
  const double first_y = -((nmy - 1) * mvy + (ncy - 1) * cvy) / 2.0;
  const int nrs = nmy * ncy;
  double* rsy = (double*)malloc(sizeof(double) * (size_t)nrs);
  for (int m = 0; m < nmy; ++m)
    for (int c = 0; c < ncy; ++c)
      rsy[m * ncy + c] = m * mvy + c * cvy + first_y;
  const double angle_interval = 2 * FO_PI / s.rsector_repeat;
  const int first_index = n_cpr - crystal_offset;
  for (int i = 0; i < first_index; ++i)
  {
    const double x = tx;
    const int io = i + crystal_offset;
    const double y = rsy[io % nrs];
    const double angle = (io / nrs) * angle_interval;
    const double ca = cos(angle), sa = sin(angle);
    xy[2 * i] = x * ca - y * sa;
    xy[2 * i + 1] = x * sa + y * ca;
  }
  for (int i = first_index; i < n_cpr; ++i)
  {
    xy[2 * i] = tx;
    xy[2 * i + 1] = rsy[i - first_index];
  }
  free(rsy);

  const int ncz = s.crystal_repeat[1], nmz = s.module_repeat[1];
  const double first_z = -((nmz - 1) * mvz + (ncz - 1) * cvz) / 2.0;
  const int nrz = nmz * ncz;
  double* ringz = (double*)malloc(sizeof(double) * (size_t)nrz);
  for (int m = 0; m < nmz; ++m)
    for (int c = 0; c < ncz; ++c)
      ringz[m * ncz + c] = m * mvz + c * cvz + first_z;
  for (int k = 0; k < 2 * n_rings - 1; ++k)
    z[k] = k % 2 == 0 ? ringz[k / 2] : (ringz[k / 2] + ringz[(k + 1) / 2]) / 2.0;
  free(ringz);
  return 0;
}

/* ---- bin to crystal pair: ProjData.cc:198-299 (axial), :301-340 (angular) ---- */
void fo_crystal_axial(const fo_proj* p, int seg, int axial, int* a1, int* a2)
{
  if (p->segment_span == 1)
  {
    if (seg == 0)
      *a1 = *a2 = 2 * axial;
    else if (seg > 0)
    {
      *a1 = 2 * (axial + seg);
      *a2 = 2 * axial;
    }
    else
    {
      *a1 = 2 * axial;
      *a2 = 2 * (axial - seg);
    }
    return;
  }
  if (seg == 0)
  {
    *a1 = *a2 = axial;
    return;
  }
  const int mid = abs(seg) * p->segment_span;
  const int h = p->half_span;
  if (axial < h)
  {
    const int rd = mid - h + axial;
    if (seg > 0) { *a1 = 2 * rd; *a2 = 0; }
    else { *a1 = 0; *a2 = 2 * rd; }
    return;
  }
  const int inv = p->n_axial[seg + p->seg_offset] - axial - 1;
  if (inv < h)
  {
    const int rd = mid - h + inv;
    const int smax = 2 * p->n_rings - 2;
    if (seg > 0) { *a1 = smax; *a2 = smax - 2 * rd; }
    else { *a1 = smax - 2 * rd; *a2 = smax; }
    return;
  }
  const int adj = axial - h;
  if (seg > 0) { *a1 = 2 * mid + adj; *a2 = adj; }
  else { *a1 = adj; *a2 = 2 * mid + adj; }
}

void fo_crystal_ang(const fo_proj* p, int view, int tang, int* c1, int* c2)
{
  const int shift = tang >= 0 ? tang / 2 : (tang - 1) / 2;
  const int odd = abs(tang) % 2;
  const int n = p->n_crystals_per_ring;
  int a = view + shift + odd;
  int b = view + p->n_views - shift;
  if (a < 0) a += n; else if (a >= n) a -= n;
  if (b < 0) b += n; else if (b >= n) b -= n;
  *c1 = a;
  *c2 = b;
}

/* ---- Siddon: Siddon.cc:20-63 (grid), :112-258 (path), :260-412 (helpers) ---- */
void fo_grid_init(fo_grid* g, const fo_vol* v, int truncate)
{
  g->nx = v->nx;
  g->ny = v->ny;
  g->nz = v->nz;
  const double vox[3] = {v->vx, v->vy, v->vz};
  for (int d = 0; d < 3; ++d) g->ext[d] = truncate ? (double)(int)vox[d] : vox[d];
  const double we = v->nx * v->vx, he = v->ny * v->vy, de = v->nz * v->vz;
  g->low[0] = v->ox - v->vx / 2;
  g->low[1] = v->oy - v->vy / 2;
  g->low[2] = v->oz - de / 2;
  g->high[0] = g->low[0] + we;
  g->high[1] = g->low[1] + he;
  g->high[2] = g->low[2] + de;
}

typedef struct
{
  double diff, amin, amax, next;
  int dir;
} fo_setup;

static int dim_setup(const fo_grid* g, int d, double c1, double c2, fo_setup* s)
{
  const double low = g->low[d], high = g->high[d];
  double diff = c2 - c1;
  if ((diff < 0 ? -diff : diff) > FO_EPS)
  {
    if (diff > 0)
    {
      s->dir = 1;
      s->amin = (low - c1) / diff;
      s->amax = (high - c1) / diff;
    }
    else
    {
      s->dir = -1;
      s->amin = (high - c1) / diff;
      s->amax = (low - c1) / diff;
    }
    s->next = 0.0;
  }
  else
  {
    if (c1 < low || c1 > high) return 0;
    diff = FO_EPS;
    s->dir = -1;
    s->amin = 0.0;
    s->amax = 1.0;
    s->next = 1.0;
  }
  s->diff = diff;
  return 1;
}

int fo_siddon(const fo_grid* g, double x1, double y1, double z1, double x2, double y2,
              double z2, int* coords, double* lengths, int cap, int* count)
{
  *count = 0;
  const double c1[3] = {x1, y1, z1}, c2[3] = {x2, y2, z2};
  fo_setup s[3];
  for (int d = 0; d < 3; ++d)
    if (!dim_setup(g, d, c1[d], c2[d], &s[d])) return 0;
  const double amin = dmax(s[0].amin, dmax(s[1].amin, dmax(s[2].amin, 0.0)));
  const double amax = dmin(s[0].amax, dmin(s[1].amax, dmin(s[2].amax, 1.0)));
  if (amin >= amax) return 0;

  double da[3];
  for (int d = 0; d < 3; ++d) da[d] = g->ext[d] / (s[d].diff < 0 ? -s[d].diff : s[d].diff);
  const double d12 = sqrt(s[0].diff * s[0].diff + s[1].diff * s[1].diff + s[2].diff * s[2].diff);

  const int nm1[3] = {g->nx - 1, g->ny - 1, g->nz - 1};
  int pos[3];
  for (int d = 0; d < 3; ++d)
  {
    int ind = (int)((c1[d] + s[d].diff * amin - g->low[d]) / g->ext[d]);
    ind = ind < nm1[d] ? ind : nm1[d];
    pos[d] = ind > 0 ? ind : 0;
  }
  double a[3];
  for (int d = 0; d < 3; ++d)
  {
    double al = s[d].next;
    if (al < 1.0)
    {
      const double len = g->low[d] + g->ext[d] * pos[d] - c1[d];
      al = len / s[d].diff;
    }
    if (s[d].dir > 0) al += da[d];
    a[d] = al;
  }

  const int row = g->nx, slice = g->nx * g->ny;
  int n = 0;
  double prev = amin;
  while (prev < amax)
  {
    const double next = dmin(amax, dmin(a[0], dmin(a[1], a[2])));
    if (pos[0] >= 0 && pos[0] <= nm1[0] && pos[1] >= 0 && pos[1] <= nm1[1] && pos[2] >= 0 &&
        pos[2] <= nm1[2])
    {
      if (n < cap)
      {
        coords[n] = pos[0] + pos[1] * row + pos[2] * slice;
        lengths[n] = (next - prev) * d12;
      }
      ++n;
    }
    for (int d = 0; d < 3; ++d)
    {
      const double dd = a[d] - next;
      if ((dd < 0 ? -dd : dd) < FO_EPS)
      {
        a[d] += da[d];
        pos[d] += s[d].dir;
      }
    }
    prev = next;
  }
  *count = n;
  return 1;
}

static void lor_ends(const fo_proj* p, const double* xy, const double* z, int seg, int view, int axial, int tang,
                     double* e);

/* ---- precision study of the traversal (not FIR code) ----
 * fo_siddon with single-precision arithmetic, to measure how often a float
 * traversal emits a voxel list different from FIR's double one:
 *   precision 1: FIR's double set-up (entry/exit alphas, first crossings,
 *                steps, start voxel), then the loop in float: alphas, their
 *                running sums, the minimum, the tie test |a - next| < 1e-5
 *                and the lengths;
 *   precision 2: the same with the set-up in float as well.
 * Returns 1 when the segment crosses the volume, like fo_siddon. */
int fo_siddon_study(const fo_grid* g, const double* e, int precision, int* coords, double* lengths, int cap,
                    int* count)
{
  *count = 0;
  int pos[3], dir[3];
  float a[3], da[3], amin_f, amax_f, d12_f;
  if (precision == 1)
  {
    fo_setup s[3];
    for (int d = 0; d < 3; ++d)
      if (!dim_setup(g, d, e[d], e[3 + d], &s[d])) return 0;
    const double amin = dmax(s[0].amin, dmax(s[1].amin, dmax(s[2].amin, 0.0)));
    const double amax = dmin(s[0].amax, dmin(s[1].amax, dmin(s[2].amax, 1.0)));
    if (amin >= amax) return 0;
    const double d12 = sqrt(s[0].diff * s[0].diff + s[1].diff * s[1].diff + s[2].diff * s[2].diff);
    const int nm1[3] = {g->nx - 1, g->ny - 1, g->nz - 1};
    for (int d = 0; d < 3; ++d)
    {
      const double dad = g->ext[d] / (s[d].diff < 0 ? -s[d].diff : s[d].diff);
      int ind = (int)((e[d] + s[d].diff * amin - g->low[d]) / g->ext[d]);
      ind = ind < nm1[d] ? ind : nm1[d];
      pos[d] = ind > 0 ? ind : 0;
      double al = s[d].next;
      if (al < 1.0) al = (g->low[d] + g->ext[d] * pos[d] - e[d]) / s[d].diff;
      if (s[d].dir > 0) al += dad;
      a[d] = (float)al;
      da[d] = (float)dad;
      dir[d] = s[d].dir;
    }
    amin_f = (float)amin;
    amax_f = (float)amax;
    d12_f = (float)d12;
  }
  else
  {
    const float eps = (float)FO_EPS;
    float diff[3], smin[3], smax[3], snext[3];
    for (int d = 0; d < 3; ++d)
    {
      const float c1 = (float)e[d], c2 = (float)e[3 + d];
      const float lo = (float)g->low[d], hi = (float)g->high[d];
      float df = c2 - c1;
      if ((df < 0 ? -df : df) > eps)
      {
        dir[d] = df > 0 ? 1 : -1;
        smin[d] = df > 0 ? (lo - c1) / df : (hi - c1) / df;
        smax[d] = df > 0 ? (hi - c1) / df : (lo - c1) / df;
        snext[d] = 0.0f;
      }
      else
      {
        if (c1 < lo || c1 > hi) return 0;
        df = eps;
        dir[d] = -1;
        smin[d] = 0.0f;
        smax[d] = 1.0f;
        snext[d] = 1.0f;
      }
      diff[d] = df;
    }
    float t = smin[2] > 0.0f ? smin[2] : 0.0f;
    t = smin[1] > t ? smin[1] : t;
    amin_f = smin[0] > t ? smin[0] : t;
    t = smax[2] < 1.0f ? smax[2] : 1.0f;
    t = smax[1] < t ? smax[1] : t;
    amax_f = smax[0] < t ? smax[0] : t;
    if (amin_f >= amax_f) return 0;
    d12_f = sqrtf(diff[0] * diff[0] + diff[1] * diff[1] + diff[2] * diff[2]);
    const int nm1[3] = {g->nx - 1, g->ny - 1, g->nz - 1};
    for (int d = 0; d < 3; ++d)
    {
      const float ext = (float)g->ext[d], lo = (float)g->low[d];
      da[d] = ext / (diff[d] < 0 ? -diff[d] : diff[d]);
      int ind = (int)(((float)e[d] + diff[d] * amin_f - lo) / ext);
      ind = ind < nm1[d] ? ind : nm1[d];
      pos[d] = ind > 0 ? ind : 0;
      float al = snext[d];
      if (al < 1.0f) al = (lo + ext * (float)pos[d] - (float)e[d]) / diff[d];
      if (dir[d] > 0) al += da[d];
      a[d] = al;
    }
  }
  const int nm1[3] = {g->nx - 1, g->ny - 1, g->nz - 1};
  const int row = g->nx, slice = g->nx * g->ny;
  const float eps = (float)FO_EPS;
  int n = 0;
  float prev = amin_f;
  while (prev < amax_f && n <= cap)
  {
    float next = a[0] < a[1] ? a[0] : a[1];
    next = a[2] < next ? a[2] : next;
    next = amax_f < next ? amax_f : next;
    if (pos[0] >= 0 && pos[0] <= nm1[0] && pos[1] >= 0 && pos[1] <= nm1[1] && pos[2] >= 0 && pos[2] <= nm1[2])
    {
      if (n < cap)
      {
        coords[n] = pos[0] + pos[1] * row + pos[2] * slice;
        lengths[n] = (double)((next - prev) * d12_f);
      }
      ++n;
    }
    for (int d = 0; d < 3; ++d)
    {
      const float dd = a[d] - next;
      if ((dd < 0 ? -dd : dd) < eps)
      {
        a[d] += da[d];
        pos[d] += dir[d];
      }
    }
    prev = next;
  }
  *count = n;
  return 1;
}

/* Precision study over the bins `bins` (n, file-order indices) of sinogram p:
 * each LOR is traversed by fo_siddon (FIR's double arithmetic) and by
 * fo_siddon_study(precision).  out[0] LORs crossing the volume, out[1] LORs
 * whose voxel lists differ (indices or length of the list), out[2] the
 * largest relative length difference on LORs with equal lists, out[3] the
 * largest and out[4] the root-mean-square relative difference of the line
 * integral of img (double sums), over crossing LORs with a non-zero
 * integral. */
static void bin_coords(const fo_proj* p, long long bin, int* seg, int* view, int* ax, int* tang)
{
  long long b = bin;
  for (int s = -p->seg_offset; s <= p->seg_offset; ++s)
  {
    const int nax = p->n_axial[s + p->seg_offset];
    const long long n = (long long)nax * p->n_views * p->n_tang_coords;
    if (b < n)
    {
      *seg = s;
      *view = (int)(b / ((long long)nax * p->n_tang_coords));
      const long long r = b - (long long)*view * nax * p->n_tang_coords;
      *ax = (int)(r / p->n_tang_coords);
      *tang = (int)(r - (long long)*ax * p->n_tang_coords) - p->tang_offset;
      return;
    }
    b -= n;
  }
}

void fo_precision_study(const fo_proj* p, const double* xy, const double* z, const fo_vol* v, int truncate,
                        const float* img, const long long* bins, long long n, int precision, double* out)
{
  fo_grid g;
  fo_grid_init(&g, v, truncate);
  const int cap = v->nx + v->ny + v->nz + 2;
  int* c1 = (int*)malloc(sizeof(int) * (size_t)cap * 2);
  double* l1 = (double*)malloc(sizeof(double) * (size_t)cap * 2);
  int* c2 = c1 + cap;
  double* l2 = l1 + cap;
  double crossing = 0, differ = 0, max_len = 0, max_line = 0, sq_line = 0, n_line = 0;
  for (long long i = 0; i < n; ++i)
  {
    int seg, view, ax, tang;
    bin_coords(p, bins[i], &seg, &view, &ax, &tang);
    double e[6];
    lor_ends(p, xy, z, seg, view, ax, tang, e);
    int n1 = 0, n2 = 0;
    const int x1 = fo_siddon(&g, e[0], e[1], e[2], e[3], e[4], e[5], c1, l1, cap, &n1);
    const int x2 = fo_siddon_study(&g, e, precision, c2, l2, cap, &n2);
    if (!x1 && !x2) continue;
    crossing += 1;
    int same = x1 == x2 && n1 == n2 && n1 <= cap;
    for (int k = 0; same && k < n1; ++k) same = c1[k] == c2[k];
    if (!same) differ += 1;
    else
      for (int k = 0; k < n1; ++k)
      {
        const double d = fabs(l2[k] - l1[k]) / (l1[k] > 0 ? l1[k] : 1.0);
        if (l1[k] > 1e-9 && d > max_len) max_len = d;
      }
    double s1 = 0, s2 = 0;
    for (int k = 0; k < n1 && k < cap; ++k) s1 += l1[k] * img[c1[k]];
    for (int k = 0; k < n2 && k < cap; ++k) s2 += l2[k] * img[c2[k]];
    if (s1 > 0)
    {
      const double r = fabs(s2 - s1) / s1;
      if (r > max_line) max_line = r;
      sq_line += r * r;
      n_line += 1;
    }
  }
  out[0] = crossing;
  out[1] = differ;
  out[2] = max_len;
  out[3] = max_line;
  out[4] = n_line > 0 ? sqrt(sq_line / n_line) : 0.0;
  free(c1);
  free(l1);
}

/* ---- projectors: projections.cc:15-92, :94-184; VolData.cc:357-385 ---- */
static long long seg_base(const fo_proj* p, int seg)
{
  long long b = 0;
  for (int s = -p->seg_offset; s < seg; ++s)
    b += (long long)p->n_axial[s + p->seg_offset] * p->n_views * p->n_tang_coords;
  return b;
}

static void lor_ends(const fo_proj* p, const double* xy, const double* z, int seg, int view,
                     int axial, int tang, double* e)
{
  int a1, a2, c1, c2;
  fo_crystal_axial(p, seg, axial, &a1, &a2);
  fo_crystal_ang(p, view, tang, &c1, &c2);
  e[0] = xy[2 * c1];
  e[1] = xy[2 * c1 + 1];
  e[2] = z[a1];
  e[3] = xy[2 * c2];
  e[4] = xy[2 * c2 + 1];
  e[5] = z[a2];
}

void fo_forward(const fo_vol* v, int truncate, const float* img, const fo_proj* p,
                const double* xy, const double* z, float* sino)
{
  fo_grid g;
  fo_grid_init(&g, v, truncate);
  const int cap = v->nx + v->ny + v->nz + 2;
  int* co = (int*)malloc(sizeof(int) * (size_t)cap);
  double* le = (double*)malloc(sizeof(double) * (size_t)cap);
  for (int seg = -p->seg_offset; seg <= p->seg_offset; ++seg)
  {
    float* out = sino + seg_base(p, seg);
    const int nax = p->n_axial[seg + p->seg_offset];
    long long b = 0;
    for (int view = 0; view < p->n_views; ++view)
      for (int ax = 0; ax < nax; ++ax)
        for (int t = -p->tang_offset; t < -p->tang_offset + p->n_tang_coords; ++t)
        {
          double e[6];
          lor_ends(p, xy, z, seg, view, ax, t, e);
          int n;
          fo_siddon(&g, e[0], e[1], e[2], e[3], e[4], e[5], co, le, cap, &n);
          float line = 0.0f;
          for (int k = 0; k < n; ++k) line = (float)((double)line + le[k] * (double)img[co[k]]);
          out[b++] = line;
        }
  }
  free(co);
  free(le);
}

/* Subset-local enumeration of LORCache.cc:10-81 and :115-133. */
void fo_backward(const fo_proj* p, const float* sino, const fo_vol* v, int truncate,
                 const double* xy, const double* z, int n_subsets, float* out)
{
  fo_grid g;
  fo_grid_init(&g, v, truncate);
  const long long nvox = (long long)v->nx * v->ny * v->nz;
  memset(out, 0, sizeof(float) * (size_t)(nvox * n_subsets));
  const int cap = v->nx + v->ny + v->nz + 2;
  int* co = (int*)malloc(sizeof(int) * (size_t)cap);
  double* le = (double*)malloc(sizeof(double) * (size_t)cap);
  const int vps = p->n_views / n_subsets;
  for (int subset = 0; subset < n_subsets; ++subset)
  {
    float* frame = out + nvox * subset;
    for (int seg = -p->seg_offset; seg <= p->seg_offset; ++seg)
    {
      const int nax = p->n_axial[seg + p->seg_offset];
      const long long bpv = (long long)nax * p->n_tang_coords;
      const long long base = seg_base(p, seg);
      for (int sv = 0; sv < vps; ++sv)
      {
        const int view = sv * n_subsets + subset;
        for (int ax = 0; ax < nax; ++ax)
          for (int ti = 0; ti < p->n_tang_coords; ++ti)
          {
            const int t = ti - p->tang_offset;
            const long long bin = view * bpv + (long long)ax * p->n_tang_coords + ti;
            const float val = sino ? sino[base + bin] : 1.0f;
            double e[6];
            lor_ends(p, xy, z, seg, view, ax, t, e);
            int n;
            fo_siddon(&g, e[0], e[1], e[2], e[3], e[4], e[5], co, le, cap, &n);
            for (int k = 0; k < n; ++k)
              frame[co[k]] = (float)((double)frame[co[k]] + le[k] * (double)val);
          }
      }
    }
  }
  free(co);
  free(le);
}

/* ---- image operations: VolData.cc:305-343, operations.cc:11-284 ---- */
void fo_em_update(long long n, float* img, float* bp, const float* sens)
{
  for (long long i = 0; i < n; ++i)
  {
    bp[i] = ((double)bp[i] > FO_EPS && (double)sens[i] > FO_EPS) ? bp[i] / sens[i] : 0.0f;
    img[i] = ((double)img[i] > FO_EPS && (double)bp[i] > FO_EPS) ? img[i] * bp[i] : 0.0f;
  }
}

static float* gauss_kernel_f(float fwhm, double vox, int* half)
{
  const float sigma = fwhm / 2.3548f;
  const int h = ((int)(6.0 * sigma / vox) + 1) / 2;
  float* k = (float*)malloc(sizeof(float) * (size_t)(2 * h + 1));
  for (int ki = -h; ki <= h; ++ki)
    k[h + ki] = (float)exp(-(ki * ki * vox * vox) / (2 * sigma * sigma));
  *half = h;
  return k;
}

static float* gauss_kernel_d(float fwhm, double vox, int* half)
{
  const double sigma = fwhm / 2.3548;
  const int h = ((int)(6.0 * sigma / vox) + 1) / 2;
  float* k = (float*)malloc(sizeof(float) * (size_t)(2 * h + 1));
  for (int ki = -h; ki <= h; ++ki)
    k[h + ki] = (float)exp(-(ki * ki * vox * vox) / (2 * sigma * sigma));
  *half = h;
  return k;
}

void fo_convolve(const fo_vol* v, float* img, const float* fwhm, float cut_radius)
{
  if (!(fwhm[0] > 0.0 && fwhm[1] > 0.0 && fwhm[2] > 0.0)) return;
  const int nx = v->nx, ny = v->ny, nz = v->nz;
  const long long n = (long long)nx * ny * nz;
  int hx, hy, hz;
  float* kx = gauss_kernel_f(fwhm[0], v->vx, &hx);
  float* ky = gauss_kernel_f(fwhm[1], v->vy, &hy);
  float* kz = gauss_kernel_d(fwhm[2], v->vz, &hz);
  float* copy = (float*)malloc(sizeof(float) * (size_t)n);
  float* im1 = (float*)calloc((size_t)n, sizeof(float));
  float* im2 = (float*)calloc((size_t)n, sizeof(float));
  memcpy(copy, img, sizeof(float) * (size_t)n);
#define IDX(i, j, k) ((long long)(i) + (long long)(j) * nx + (long long)(k) * nx * ny)
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i)
      {
        float sum = 0.0f, norm = 0.0f;
        for (int ki = -hx; ki <= hx; ++ki)
          if (i + ki >= 0 && i + ki < nx)
          {
            const float kv = kx[hx + ki];
            sum += kv * img[IDX(i + ki, j, k)];
            norm += kv;
          }
        if (norm > 0.0) im1[IDX(i, j, k)] = sum / norm;
      }
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i)
      {
        float sum = 0.0f, norm = 0.0f;
        for (int ki = -hy; ki <= hy; ++ki)
          if (j + ki >= 0 && j + ki < ny)
          {
            const float kv = ky[hy + ki];
            sum += kv * im1[IDX(i, j + ki, k)];
            norm += kv;
          }
        if (norm > 0.0) im2[IDX(i, j, k)] = sum / norm;
      }
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i)
      {
        float sum = 0.0f, norm = 0.0f;
        for (int ki = -hz; ki <= hz; ++ki)
          if (k + ki >= 0 && k + ki < nz)
          {
            const float kv = kz[hz + ki];
            sum += kv * im2[IDX(i, j, k + ki)];
            norm += kv;
          }
        if (norm > 0.0) img[IDX(i, j, k)] = sum / norm;
      }
  if (cut_radius > 0.0)
  {
    const float f = fwhm[0] > fwhm[1] ? fwhm[0] : fwhm[1];
    const double sw = nx * v->vx, sh = ny * v->vy;
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j)
        for (int i = 0; i < nx; ++i)
        {
          const double px = i * v->vx + v->vx / 2.0 - sw / 2.0;
          const double py = j * v->vy + v->vy / 2.0 - sh / 2.0;
          if (sqrt(px * px + py * py) >= cut_radius - 5.0 * f) img[IDX(i, j, k)] = copy[IDX(i, j, k)];
        }
  }
#undef IDX
  free(kx);
  free(ky);
  free(kz);
  free(copy);
  free(im1);
  free(im2);
}

void fo_cut_circle(const fo_vol* v, float* img, float cut_radius)
{
  if (!(cut_radius > 0.0)) return;
  const double sw = v->nx * v->vx, sh = v->ny * v->vy;
  for (int k = 0; k < v->nz; ++k)
    for (int j = 0; j < v->ny; ++j)
      for (int i = 0; i < v->nx; ++i)
      {
        const double px = i * v->vx + v->vx / 2.0 - sw / 2.0;
        const double py = j * v->vy + v->vy / 2.0 - sh / 2.0;
        if (sqrt(px * px + py * py) > cut_radius)
          img[i + (long long)j * v->nx + (long long)k * v->nx * v->ny] = 0.0f;
      }
}

void fo_apply_mask(long long n, float* img, const float* mask)
{
  for (long long i = 0; i < n; ++i)
    if (mask[i] <= 0) img[i] = 0.0f;
}

void fo_hu_to_mu(long long n, float* img)
{
  const float water = 0.0096f, thousand = 0.015f;
  const float s1 = water / (float)1000.0, s2 = (thousand - water) / (float)1000.0;
  for (long long i = 0; i < n; ++i)
  {
    if (img[i] <= -1000.0)
      img[i] = 0.0f;
    else if (img[i] <= 0.0)
    {
      img[i] *= s1;
      img[i] += water;
    }
    else
    {
      img[i] *= s2;
      img[i] += water;
    }
  }
}

void fo_exponential(long long n, float* sino)
{
  for (long long i = 0; i < n; ++i) sino[i] = (double)sino[i] > FO_EPS ? expf(sino[i]) : 1.0f;
}

void fo_proj_multiply(long long n, float* a, const float* b)
{
  for (long long i = 0; i < n; ++i)
    a[i] = ((double)a[i] > FO_EPS && (double)b[i] > FO_EPS) ? a[i] * b[i] : 0.0f;
}

/* ---- OSEM: reconAlgos.cc:11-59 (getLine), :63-201 (loop) ---- */
/* The OSEM loop of reconAlgos.cc:63-201.  With mult (per-bin multiplicative
 * factors), the ordinary-Poisson model: estimate m * line + bias, and the
 * backprojected value m * measured / estimate.  With psf, the resolution-modelling
 * variant that OSEM_ResoReco (reconAlgos.cc:203-367) intends, corrected: the
 * Gaussian B = operations::convolve(fwhm, cutRadius) sits inside the system
 * model.  Each sub-iteration projects B x (FIR projects x, :296), blurs the
 * backprojection (:300-304), and divides it by the blurred sensitivity of
 * the subset before the usual EM update (FIR divides the image, :323);
 * every sensitivity frame is blurred once before the loop. */
static void osem_loop(const fo_proj* p, const float* sino, const float* mult, const float* bias, const fo_vol* v,
                      int truncate, const double* xy, const double* z, float* img, const float* sens,
                      const fo_osem_params* prm, int psf)
{
  fo_grid g;
  fo_grid_init(&g, v, truncate);
  const long long nvox = (long long)v->nx * v->ny * v->nz;
  float* bp = (float*)calloc((size_t)nvox, sizeof(float));
  const int cap = v->nx + v->ny + v->nz + 2;
  int* co = (int*)malloc(sizeof(int) * (size_t)cap);
  double* le = (double*)malloc(sizeof(double) * (size_t)cap);
  const int conv = prm->convolution_interval > 0 && prm->fwhm[0] > 0.0 && prm->fwhm[1] > 0.0 &&
                   prm->fwhm[2] > 0.0;
  const int nsub = prm->n_subsets, vps = p->n_views / nsub;
  float* blur = NULL;
  float* sens_b = NULL;
  if (psf)
  {
    blur = (float*)malloc(sizeof(float) * (size_t)nvox);
    sens_b = (float*)malloc(sizeof(float) * (size_t)(nvox * nsub));
    memcpy(sens_b, sens, sizeof(float) * (size_t)(nvox * nsub));
    for (int s = 0; s < nsub; ++s) fo_convolve(v, sens_b + nvox * s, prm->fwhm, prm->cut_radius);
  }
  fo_cut_circle(v, img, prm->cut_radius);
  for (int iter = 0; iter < prm->n_iterations; ++iter)
    for (int subset = 0; subset < nsub; ++subset)
    {
      const int subiter = iter * nsub + subset + 1;
      const float* model = img;
      if (psf)
      {
        memcpy(blur, img, sizeof(float) * (size_t)nvox);
        fo_convolve(v, blur, prm->fwhm, prm->cut_radius);
        model = blur;
      }
      for (int seg = -p->seg_offset; seg <= p->seg_offset; ++seg)
      {
        const int nax = p->n_axial[seg + p->seg_offset];
        const long long bpv = (long long)nax * p->n_tang_coords;
        const long long base = seg_base(p, seg);
        for (int sv = 0; sv < vps; ++sv)
        {
          const int view = sv * nsub + subset;
          for (int ax = 0; ax < nax; ++ax)
            for (int ti = 0; ti < p->n_tang_coords; ++ti)
            {
              const long long bin = base + view * bpv + (long long)ax * p->n_tang_coords + ti;
              double e[6];
              lor_ends(p, xy, z, seg, view, ax, ti - p->tang_offset, e);
              int n;
              const int crosses = fo_siddon(&g, e[0], e[1], e[2], e[3], e[4], e[5], co, le, cap, &n);
              float line = 0.0f;
              if (crosses)
                for (int k = 0; k < n; ++k) line = (float)((double)line + le[k] * (double)model[co[k]]);
              if (mult) line = line * mult[bin];
              if (bias) line += bias[bin];
              if ((double)line > FO_EPS)
              {
                float ratio = sino[bin] / line;
                if (mult) ratio = ratio * mult[bin];
                for (int k = 0; k < n; ++k) bp[co[k]] = (float)((double)bp[co[k]] + le[k] * (double)ratio);
              }
            }
        }
      }
      if (psf) fo_convolve(v, bp, prm->fwhm, prm->cut_radius);
      fo_em_update(nvox, img, bp, (psf ? sens_b : sens) + nvox * subset);
      if (conv && subiter % prm->convolution_interval == 0) fo_convolve(v, img, prm->fwhm, prm->cut_radius);
      fo_cut_circle(v, img, prm->cut_radius);
      memset(bp, 0, sizeof(float) * (size_t)nvox);
    }
  free(blur);
  free(sens_b);
  free(bp);
  free(co);
  free(le);
}

void fo_osem(const fo_proj* p, const float* sino, const float* bias, const fo_vol* v, int truncate,
             const double* xy, const double* z, float* img, const float* sens, const fo_osem_params* prm)
{
  osem_loop(p, sino, NULL, bias, v, truncate, xy, z, img, sens, prm, 0);
}

void fo_osem_weighted(const fo_proj* p, const float* sino, const float* mult, const float* bias, const fo_vol* v,
                      int truncate, const double* xy, const double* z, float* img, const float* sens,
                      const fo_osem_params* prm)
{
  osem_loop(p, sino, mult, bias, v, truncate, xy, z, img, sens, prm, 0);
}

void fo_osem_psf(const fo_proj* p, const float* sino, const float* bias, const fo_vol* v, int truncate,
                 const double* xy, const double* z, float* img, const float* sens, const fo_osem_params* prm)
{
  const int psf = prm->fwhm[0] > 0.0 && prm->fwhm[1] > 0.0 && prm->fwhm[2] > 0.0;
  osem_loop(p, sino, NULL, bias, v, truncate, xy, z, img, sens, prm, psf);
}

/* reconAlgos::OSEM_ResoReco as FIR runs it (reconAlgos.cc:203-367): the
 * initial cut (:229); all n_sens_frames frames of the sensitivity filtered in
 * place (:232-236; operations::convolve filters every frame,
 * operations.cc:77-187); per sub-iteration the ratio backprojection of
 * the unfiltered image (:270-312), the backprojection filtered (:315-319),
 * img /= sens[subset] and img *= bp with VolData's gates (:321-326;
 * VolData.cc:305-343), the post-filter (:333-341) and the cut (:344).  The
 * filtered copy `blur` (:239, :264-268, :350-353) is never read and is left
 * out. */
void fo_osem_reso_reco(const fo_proj* p, const float* sino, const float* bias, const fo_vol* v, int truncate,
                       const double* xy, const double* z, float* img, float* sens, int n_sens_frames,
                       const fo_osem_params* prm)
{
  fo_grid g;
  fo_grid_init(&g, v, truncate);
  const long long nvox = (long long)v->nx * v->ny * v->nz;
  float* bp = (float*)calloc((size_t)nvox, sizeof(float));
  const int cap = v->nx + v->ny + v->nz + 2;
  int* co = (int*)malloc(sizeof(int) * (size_t)cap);
  double* le = (double*)malloc(sizeof(double) * (size_t)cap);
  const int conv = prm->convolution_interval > 0 && prm->fwhm[0] > 0.0 && prm->fwhm[1] > 0.0 &&
                   prm->fwhm[2] > 0.0;
  const int nsub = prm->n_subsets, vps = p->n_views / nsub;
  fo_cut_circle(v, img, prm->cut_radius);
  for (int f = 0; f < n_sens_frames; ++f) fo_convolve(v, sens + nvox * f, prm->fwhm, prm->cut_radius);
  for (int iter = 0; iter < prm->n_iterations; ++iter)
    for (int subset = 0; subset < nsub; ++subset)
    {
      const int subiter = iter * nsub + subset + 1;
      memset(bp, 0, sizeof(float) * (size_t)nvox);
      for (int seg = -p->seg_offset; seg <= p->seg_offset; ++seg)
      {
        const int nax = p->n_axial[seg + p->seg_offset];
        const long long bpv = (long long)nax * p->n_tang_coords;
        const long long base = seg_base(p, seg);
        for (int sv = 0; sv < vps; ++sv)
        {
          const int view = sv * nsub + subset;
          for (int ax = 0; ax < nax; ++ax)
            for (int ti = 0; ti < p->n_tang_coords; ++ti)
            {
              const long long bin = base + view * bpv + (long long)ax * p->n_tang_coords + ti;
              double e[6];
              lor_ends(p, xy, z, seg, view, ax, ti - p->tang_offset, e);
              int n;
              const int crosses = fo_siddon(&g, e[0], e[1], e[2], e[3], e[4], e[5], co, le, cap, &n);
              float line = 0.0f;
              if (crosses)
                for (int k = 0; k < n; ++k) line = (float)((double)line + le[k] * (double)img[co[k]]);
              if (bias) line += bias[bin];
              if ((double)line > FO_EPS)
              {
                const float ratio = sino[bin] / line;
                for (int k = 0; k < n; ++k) bp[co[k]] = (float)((double)bp[co[k]] + le[k] * (double)ratio);
              }
            }
        }
      }
      fo_convolve(v, bp, prm->fwhm, prm->cut_radius);
      const float* sf = sens + nvox * subset;
      for (long long i = 0; i < nvox; ++i)
      {
        float x = img[i];
        x = ((double)x > FO_EPS && (double)sf[i] > FO_EPS) ? x / sf[i] : 0.0f;
        x = ((double)x > FO_EPS && (double)bp[i] > FO_EPS) ? x * bp[i] : 0.0f;
        img[i] = x;
      }
      if (conv && subiter % prm->convolution_interval == 0) fo_convolve(v, img, prm->fwhm, prm->cut_radius);
      fo_cut_circle(v, img, prm->cut_radius);
    }
  free(bp);
  free(co);
  free(le);
}

/* ProjData::getBinCoordinates (ProjData.cc:342-479): the sinogram bin of the
 * LOR between (ring1, crystal1) and (ring2, crystal2), in integer arithmetic
 * with C's truncating division.  Returns 0 when the LOR lies outside the
 * allocated segments or tangential range. */
int fo_bin_coordinates(const fo_proj* p, int r1, int c1, int r2, int c2, int* seg, int* view, int* axial,
                       int* tang)
{
  const int n = p->n_crystals_per_ring;
  int aseg = r1 > r2 ? r1 - r2 : r2 - r1;
  if (aseg > p->max_ring_diff) return 0;
  const int sum = c1 + c2;
  const int s1 = (sum >= n / 2 && sum < 3 * n / 2) ? -1 : 1;
  const int t = s1 * ((c2 > c1 ? c2 - c1 : c1 - c2) - n / 2);
  if (t < -p->tang_offset || t >= -p->tang_offset + p->n_tang_coords) return 0;
  int ax;
  if (p->segment_span == 1)
    ax = (r1 + r2 - aseg) / 2;
  else
  {
    const int central = aseg <= p->half_span;
    aseg = central ? 0 : 1 + (aseg - p->half_span - 1) / p->segment_span;
    const int m = central ? 0 : 1 + p->half_span + (aseg - 1) * p->segment_span;
    ax = r1 + r2 - m;
  }
  const int v = ((sum + n / 2) % n) / 2;
  int sg = aseg;
  if (sg != 0)
  {
    const int s2 = c1 < c2 ? 1 : -1;
    const int at = t < 0 ? -t : t;
    const int u = at % 2 == 0 ? -t / 2 : -(t - 1) / 2;
    int k1 = c1 - s1 * s2 * u, k2 = c2 + s1 * s2 * u;
    if (k1 >= n) k1 -= n; else if (k1 < 0) k1 += n;
    if (k2 >= n) k2 -= n; else if (k2 < 0) k2 += n;
    sg = sg * (r1 < r2 ? -1 : 1) * (k1 < k2 ? 1 : -1);
  }
  *seg = sg;
  *view = v;
  *axial = ax;
  *tang = t;
  return 1;
}

/* ProjData::rebinWeight (ProjData.cc:541-615): for span > 1, every bin of an
 * axial position that merges w > 1 ring differences of one ring sum is
 * multiplied by (float)(1.0 / w), serially in FIR's loop order. */
void fo_rebin_weight(const fo_proj* p, float* sino)
{
  if (p->segment_span == 1) return;
  const int nr = p->n_rings, span = p->segment_span;
  for (int rs = 0; rs <= 2 * (nr - 1); ++rs)
  {
    int lmd = rs <= nr - 1 ? rs : 2 * (nr - 1) - rs;
    if (lmd > p->max_ring_diff) lmd = p->max_ring_diff;
    if ((rs + lmd) % 2) --lmd;
    int seg = -p->seg_offset - 1, next = -p->max_ring_diff - 1;
    while (next < -lmd)
    {
      ++seg;
      next += span;
    }
    int w = 1;
    for (int rd = -lmd; rd <= lmd; rd += 2)
    {
      if (rd == lmd || rd + 1 >= next)
      {
        if (w > 1)
        {
          const int aseg = seg < 0 ? -seg : seg;
          const int ax = seg == 0 ? rs : rs - (span + 1) / 2 - (aseg - 1) * span;
          const float f = (float)(1.0 / w);
          const int nax = p->n_axial[seg + p->seg_offset];
          const long long bpv = (long long)nax * p->n_tang_coords;
          const long long base = seg_base(p, seg);
          for (int view = 0; view < p->n_views; ++view)
            for (int ti = 0; ti < p->n_tang_coords; ++ti)
            {
              const long long bin = base + view * bpv + (long long)ax * p->n_tang_coords + ti;
              sino[bin] = sino[bin] * f;
            }
        }
        w = 1;
        ++seg;
        next += span;
      }
      else
        ++w;
    }
  }
}
