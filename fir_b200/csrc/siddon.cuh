// Device-side geometry and the Siddon traversal of FIR (src_lib/Siddon.cc).
//
// The traversal reproduces FIR's double-precision arithmetic operation by
// operation: every add, multiply, divide and square root is an explicit
// round-to-nearest intrinsic (never fused into an FMA), extents, planes and
// tie tolerance are FIR's, and the loop visits and emits exactly the voxels
// FIR's computePath emits, with the same lengths.  The voxel index lists are
// therefore bit-identical to FIR's.
//
// Kernels call the traversal from every lane (lanes without a LOR pass
// go = false) and never return before it, so a warp's 32 LORs step through
// their loops together; between two traversals of one lane the kernel
// re-converges the warp with __syncwarp().
#pragma once

#include <cstdint>

namespace fir
{
constexpr double kEps = 0.00001;   // macros.h:8
constexpr int kMaxSegments = 255;  // 2*128-1 segments: up to 128 rings at span 1

// Volume grid as the traversal sees it (Siddon.cc:20-63).
struct Grid
{
  int nx, ny, nz, nxy;
  int guard;       // bound on traversal steps: planes crossed in all dimensions + margin
  int exact_only;  // 1: always FIR's subtraction tie test, bounded by guard (testing aid)
  double ext[3];   // step sizes: FIR's int-truncated extents, or the real ones
  double low[3];   // border planes: x,y = offset - voxel/2, z = offset - depth/2
  double high[3];  // low + n * voxel (real voxel extents, as in FIR)
  double rext[3];  // RN(1 / ext)
};

// Sinogram enumeration for one launch.  Bins are enumerated segment by
// segment in FIR's order; inside a segment, subset-local index r maps to
// view = (r / binsPerView) * nSubsets + subset (LORCache.cc:115-133).
struct Sino
{
  int n_rings, n_cpr, span, half_span;
  int n_segments, seg_offset, tang_offset, n_views, n_tang;
  int n_subsets, subset;
  int n_enum;                          // bins enumerated by this launch
  int seg_base[kMaxSegments + 1];      // first flat bin of each segment (file order)
  int enum_base[kMaxSegments + 1];     // first enumerated index of each segment
  int n_axial[kMaxSegments];
  // null, or a compacted enumeration: thread i < *list_n takes the enumerated
  // index list[i] (ascending), so that skipped bins take no lanes
  const int* list;
  const int* list_n;
};

struct Tables
{
  const double2* xy;  // crystal centres of one ring (ScannerData.cc:248-329)
  const double* z;    // slice centres, 2*nRings-1 (ScannerData.cc:331-377)
};

struct Lor
{
  int bin;     // flat bin index (file order)
  int seg, view, axial, tang;
};

__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }
// RN(a / b) from rb = RN(1 / b).  q = RN(a rb) is within two ulps of a / b;
// a correction by the remainder a - b q (one fused multiply-add) makes it
// faithful, and a second correction then rounds it correctly by Markstein's
// theorem (P. Markstein, IBM J. Res. Develop. 34(1), 1990: with y = RN(1/b)
// and q faithful, RN(q + y (a - b q)) = RN(a / b)).  The theorem needs finite
// operands far from overflow and underflow, as the traversal's finite ones
// are.  An infinite operand makes a remainder NaN (inf * 0 or inf - inf);
// for those operands RN(a rb) itself is the IEEE quotient (finite / inf =
// signed 0, inf / finite = signed inf, inf / inf and NaN give NaN), and it
// is returned instead.
__device__ __forceinline__ double ddiv_r(double a, double b, double rb)
{
  const double q0 = __dmul_rn(a, rb);
  double r = __fma_rn(-b, q0, a);
  double q = __fma_rn(r, rb, q0);
  r = __fma_rn(-b, q, a);
  q = __fma_rn(r, rb, q);
  return q == q ? q : q0;
}

// Enumerated index -> bin coordinates, for subset `subset` of s.n_subsets
// (the enumeration bases depend only on the number of subsets).
__device__ __forceinline__ Lor decode_bin(const Sino& s, int i, int subset)
{
  int lo = 0, hi = s.n_segments;
  while (hi - lo > 1)
  {
    const int mid = (lo + hi) >> 1;
    if (s.enum_base[mid] <= i)
      lo = mid;
    else
      hi = mid;
  }
  const int r = i - s.enum_base[lo];
  const int nax = s.n_axial[lo];
  const int bpv = nax * s.n_tang;
  const int sv = r / bpv;
  const int rem = r - sv * bpv;
  const int ax = rem / s.n_tang;
  Lor l;
  l.view = sv * s.n_subsets + subset;
  l.seg = lo - s.seg_offset;
  l.axial = ax;
  l.tang = rem - ax * s.n_tang - s.tang_offset;
  l.bin = s.seg_base[lo] + l.view * bpv + rem;
  return l;
}

__device__ __forceinline__ Lor decode_bin(const Sino& s, int i) { return decode_bin(s, i, s.subset); }

// The enumerated index that thread i traces: i itself, or the i-th entry of
// the compacted list; valid is false past the end of either.
__device__ __forceinline__ int enum_index(const Sino& s, int i, bool& valid)
{
  if (s.list == nullptr)
  {
    valid = i < s.n_enum;
    return i;
  }
  valid = i < __ldg(s.list_n);
  return valid ? __ldg(s.list + i) : 0;
}

// ProjData::getCrystalAxialCoord (ProjData.cc:198-299): slice indices.
__device__ __forceinline__ void crystal_axial(const Sino& s, int seg, int axial, int& a1, int& a2)
{
  if (s.span == 1)
  {
    if (seg == 0)
    {
      a1 = a2 = 2 * axial;
    }
    else if (seg > 0)
    {
      a1 = 2 * (axial + seg);
      a2 = 2 * axial;
    }
    else
    {
      a1 = 2 * axial;
      a2 = 2 * (axial - seg);
    }
    return;
  }
  if (seg == 0)
  {
    a1 = a2 = axial;
    return;
  }
  const int aseg = seg < 0 ? -seg : seg;
  const int mid = aseg * s.span;
  const int h = s.half_span;
  if (axial < h)
  {
    const int rd = mid - h + axial;
    a1 = seg > 0 ? 2 * rd : 0;
    a2 = seg > 0 ? 0 : 2 * rd;
    return;
  }
  const int inv = s.n_axial[seg + s.seg_offset] - axial - 1;
  if (inv < h)
  {
    const int rd = mid - h + inv;
    const int smax = 2 * s.n_rings - 2;
    a1 = seg > 0 ? smax : smax - 2 * rd;
    a2 = seg > 0 ? smax - 2 * rd : smax;
    return;
  }
  const int adj = axial - h;
  a1 = seg > 0 ? 2 * mid + adj : adj;
  a2 = seg > 0 ? adj : 2 * mid + adj;
}

// ProjData::getCrystalAngCoord (ProjData.cc:301-340).
__device__ __forceinline__ void crystal_ang(const Sino& s, int view, int tang, int& c1, int& c2)
{
  const int shift = tang >= 0 ? tang / 2 : (tang - 1) / 2;
  const int odd = (tang < 0 ? -tang : tang) & 1;
  int a = view + shift + odd;
  int b = view + s.n_views - shift;
  if (a < 0)
    a += s.n_cpr;
  else if (a >= s.n_cpr)
    a -= s.n_cpr;
  if (b < 0)
    b += s.n_cpr;
  else if (b >= s.n_cpr)
    b -= s.n_cpr;
  c1 = a;
  c2 = b;
}

__device__ __forceinline__ void lor_ends(const Sino& s, const Tables& t, const Lor& l, double e[6])
{
  int a1, a2, c1, c2;
  crystal_axial(s, l.seg, l.axial, a1, a2);
  crystal_ang(s, l.view, l.tang, c1, c2);
  const double2 p1 = __ldg(t.xy + c1);
  const double2 p2 = __ldg(t.xy + c2);
  e[0] = p1.x;
  e[1] = p1.y;
  e[2] = __ldg(t.z + a1);
  e[3] = p2.x;
  e[4] = p2.y;
  e[5] = __ldg(t.z + a2);
}

// ProjData::getBinCoordinates (ProjData.cc:342-479): the bin (seg, view,
// axial, tang) of the LOR between crystal c1 of ring r1 and crystal c2 of
// ring r2; false when the LOR lies outside the allocated segments or
// tangential range.  Integer arithmetic with truncating division, as FIR's.
__device__ __forceinline__ bool bin_of_crystals(const Sino& s, int max_ring_diff, int r1, int c1, int r2, int c2,
                                                int out[4])
{
  const int n = s.n_cpr;
  int aseg = r1 > r2 ? r1 - r2 : r2 - r1;
  if (aseg > max_ring_diff)
  {
    return false;
  }
  const int sum = c1 + c2;
  const int s1 = (sum >= n / 2 && sum < 3 * n / 2) ? -1 : 1;
  const int t = s1 * ((c2 > c1 ? c2 - c1 : c1 - c2) - n / 2);
  if (t < -s.tang_offset || t >= -s.tang_offset + s.n_tang)
  {
    return false;
  }
  int ax;
  if (s.span == 1)
  {
    ax = (r1 + r2 - aseg) / 2;
  }
  else
  {
    const bool central = aseg <= s.half_span;
    aseg = central ? 0 : 1 + (aseg - s.half_span - 1) / s.span;
    const int m = central ? 0 : 1 + s.half_span + (aseg - 1) * s.span;
    ax = r1 + r2 - m;
  }
  int seg = aseg;
  if (seg != 0)
  {
    // the crystals of the parallel LOR nearest the axis (tang 0 or 1) decide
    // the sign together with the ring order
    const int s2 = c1 < c2 ? 1 : -1;
    const int at = t < 0 ? -t : t;
    const int u = at % 2 == 0 ? -t / 2 : -(t - 1) / 2;
    int k1 = c1 - s1 * s2 * u;
    int k2 = c2 + s1 * s2 * u;
    k1 = k1 >= n ? k1 - n : (k1 < 0 ? k1 + n : k1);
    k2 = k2 >= n ? k2 - n : (k2 < 0 ? k2 + n : k2);
    seg = seg * (r1 < r2 ? -1 : 1) * (k1 < k2 ? 1 : -1);
  }
  out[0] = seg;
  out[1] = ((sum + n / 2) % n) / 2;
  out[2] = ax;
  out[3] = t;
  return true;
}

// State of one path.  The voxel is tracked as its linear index plus, per
// dimension, the number of further advances that keep the index inside the
// volume: FIR's checkIndices (Siddon.cc:394-404) holds exactly while all
// three counts are non-negative, because each index moves monotonically.
struct Walk
{
  double a[3];   // alpha of the next plane crossing in each dimension
  double da[3];  // alpha between neighbouring planes
  int left[3];   // advances left before the index leaves the volume
  int step[3];   // change of the linear index per advance
  int c;         // linear index of the current voxel
  int tr;        // 1: index of the layout with x and y exchanged, [z][x][y]
  double amin, amax, d12;
};

// Siddon::computePath setup (Siddon.cc:112-203 with dimSetup :260-317,
// getEntryExit :319-334, getStartInd :336-350, prepareDim :352-377).
// Returns false when the segment misses the volume.  With transpose the
// linear index is that of the image with x and y exchanged ([z][x][y]); the
// traversal itself is the same.
__device__ __forceinline__ bool siddon_setup(const Grid& g, const double e[6], Walk& w, bool transpose = false)
{
  double diff[3], smin[3], smax[3], snext[3];
  int dir[3];
#pragma unroll
  for (int d = 0; d < 3; ++d)
  {
    const double c1 = e[d], c2 = e[3 + d];
    const double lo = g.low[d], hi = g.high[d];
    double df = dsub(c2, c1);
    if (fabs(df) > kEps)
    {
      const double rdf = __drcp_rn(df);
      if (df > 0)
      {
        dir[d] = 1;
        smin[d] = ddiv_r(dsub(lo, c1), df, rdf);
        smax[d] = ddiv_r(dsub(hi, c1), df, rdf);
      }
      else
      {
        dir[d] = -1;
        smin[d] = ddiv_r(dsub(hi, c1), df, rdf);
        smax[d] = ddiv_r(dsub(lo, c1), df, rdf);
      }
      snext[d] = 0.0;
    }
    else
    {
      if (c1 < lo || c1 > hi)
      {
        return false;
      }
      df = kEps;
      dir[d] = -1;
      smin[d] = 0.0;
      smax[d] = 1.0;
      snext[d] = 1.0;
    }
    diff[d] = df;
  }
  // MAX(a, MAX(b, MAX(c, 0))) and MIN(a, MIN(b, MIN(c, 1))), macros.h:4-5
  double t = smin[2] > 0.0 ? smin[2] : 0.0;
  t = smin[1] > t ? smin[1] : t;
  w.amin = smin[0] > t ? smin[0] : t;
  t = smax[2] < 1.0 ? smax[2] : 1.0;
  t = smax[1] < t ? smax[1] : t;
  w.amax = smax[0] < t ? smax[0] : t;
  if (w.amin >= w.amax)
  {
    return false;
  }
  const int n[3] = {g.nx, g.ny, g.nz};
  const int stride[3] = {transpose ? g.ny : 1, transpose ? 1 : g.nx, g.nxy};
  w.tr = transpose ? 1 : 0;
  double rdiff[3];
#pragma unroll
  for (int d = 0; d < 3; ++d)
  {
    // RN is symmetric, so ext / |diff| = |RN(ext / diff)|
    rdiff[d] = __drcp_rn(diff[d]);
    w.da[d] = fabs(ddiv_r(g.ext[d], diff[d], rdiff[d]));
  }
  w.d12 = __dsqrt_rn(dadd(dadd(dmul(diff[0], diff[0]), dmul(diff[1], diff[1])), dmul(diff[2], diff[2])));
  w.c = 0;
#pragma unroll
  for (int d = 0; d < 3; ++d)
  {
    int ind = __double2int_rz(ddiv_r(dsub(dadd(e[d], dmul(diff[d], w.amin)), g.low[d]), g.ext[d], g.rext[d]));
    ind = ind < n[d] - 1 ? ind : n[d] - 1;
    ind = ind > 0 ? ind : 0;
    double al = snext[d];
    if (al < 1.0)
    {
      al = ddiv_r(dsub(dadd(g.low[d], dmul(g.ext[d], (double)ind)), e[d]), diff[d], rdiff[d]);
    }
    if (dir[d] > 0)
    {
      al = dadd(al, w.da[d]);
    }
    w.a[d] = al;
    w.left[d] = dir[d] > 0 ? n[d] - 1 - ind : ind;
    w.step[d] = dir[d] * stride[d];
    w.c += ind * stride[d];
  }
  return true;
}

// MIN macro of macros.h:4 on doubles (a compare and a select; cheaper on the
// GPU than fmin, which must also order NaNs and signed zeros).
__device__ __forceinline__ double min_of(double a, double b) { return a < b ? a : b; }

// The computePath loop (Siddon.cc:207-252) from the state after setup.
//
// FIR stores an element only while checkIndices holds (Siddon.cc:394-404)
// and keeps stepping until alpha reaches alphaMax.  The indices start inside
// the volume (getStartInd clamps them) and each moves monotonically, so once
// one has left the volume no later step stores anything: the loop stops
// there, and every step it takes stores its element.
//
// Tie rule (updateDim, Siddon.cc:379-392): dimension d advances when
// |alpha_d - alphaNext| < EPS, i.e. rn(alpha_d - next) < EPS since
// alpha_d >= next.  kFastTie uses the equivalent alpha_d < ru(next + EPS),
// which is exact whenever next >= EPS: for next <= alpha_d <= 2 next the
// subtraction is exact (Sterbenz), so the test is the real comparison
// alpha_d < next + EPS, which for a double alpha_d is alpha_d < ru(next +
// EPS); for alpha_d > 2 next both tests are false.  The fast form costs one
// add per step instead of three.  walk_step is one step of the loop.
// One step from prev: emits the element and advances the dimensions that
// cross at the next alpha; returns that alpha.
template<bool kFastTie, class Emit>
__device__ __forceinline__ double walk_step(Walk& w, double prev, bool& more, Emit&& emit)
{
  double next;
  if (kFastTie)
  {
    // No alpha is NaN here, so MIN's operand order does not matter, and
    // next < alphaMax (the loop test on the new prev) is the compare that
    // picks next: m when m < alphaMax, else alphaMax.
    const double m = min_of(w.a[0], min_of(w.a[1], w.a[2]));
    more = m < w.amax;
    next = more ? m : w.amax;
  }
  else
  {
    // MIN(alphaMax, MIN(ax, MIN(ay, az))) in FIR's order, which also fixes
    // which operand wins when an alpha is NaN (non-finite end points).
    next = min_of(w.amax, min_of(w.a[0], min_of(w.a[1], w.a[2])));
    more = next < w.amax;
  }
  emit(true, w.c, dmul(dsub(next, prev), w.d12));
  const double thr = kFastTie ? __dadd_ru(next, kEps) : 0.0;
#pragma unroll
  for (int d = 0; d < 3; ++d)
  {
    if (kFastTie ? w.a[d] < thr : dsub(w.a[d], next) < kEps)
    {
      w.a[d] = dadd(w.a[d], w.da[d]);
      w.c += w.step[d];
      w.left[d] -= 1;
    }
  }
  more = more && (w.left[0] | w.left[1] | w.left[2]) >= 0;
  return next;
}

// Advances left in each dimension, from the linear index (every index is
// inside the volume when this is called).
__device__ __forceinline__ void left_from_index(const Grid& g, Walk& w)
{
  const int z = w.c / g.nxy;
  const int rest = w.c - z * g.nxy;
  const int slow = rest / (w.tr ? g.ny : g.nx);
  const int fast = rest - slow * (w.tr ? g.ny : g.nx);
  const int idx[3] = {w.tr ? slow : fast, w.tr ? fast : slow, z};
  const int n[3] = {g.nx, g.ny, g.nz};
#pragma unroll
  for (int d = 0; d < 3; ++d)
  {
    w.left[d] = w.step[d] > 0 ? n[d] - 1 - idx[d] : idx[d];
  }
}

// With the fast tie form every alpha is finite or +inf and >= EPS, and
// alphaMax <= 1, so every step either advances the dimension that attains
// the minimum (using up one of its finitely many advances) or reaches
// alphaMax: the loop ends without a step bound.
//
// Most steps are far from any index leaving the volume, and those need
// neither the advance counts nor the alphaMax select.  Dimension d leaves
// the volume at its (left_d + 1)-th crossing, at alpha X_d = a_d + left_d
// da_d (accumulated by repeated addition; the closed form differs from the
// sum by at most (left_d + 2) ulp(X_d), far below X_d 2^-20).  A step
// advances that crossing only if X_d < ru(next + EPS), so while next <
// X_d - EPS - X_d 2^-20 for every d, and next < alphaMax, no index leaves
// and next is the minimum alpha.  Those steps run first without the
// bookkeeping; the advance counts are then rebuilt from the linear index
// and the checked steps finish the walk.
//
// The unchecked steps run in pairs behind one test.  A step moves the
// minimum by at most the largest step `big` of the dimensions whose next
// crossing lies below 1 (the one attaining the minimum advances by its
// step, rounded; the others stay), and a dimension whose crossing is at or
// beyond 1 never attains a minimum below end <= alphaMax <= 1 again, since
// alphas only grow.  So a pair whose first minimum lies below end - big -
// 4 EPS has its second one below end too.  The steps left before end run
// singly.
//
// A dimension advances by adding a selected addend: its step when the tie
// test holds, else the subnormal double whose low word is the step's (its
// high word zeroed), which rounding absorbs: rn(a + s) = a for every alpha
// of these steps (a >= EPS, s < 2^-1042).  The running sums are therefore
// FIR's, and one select of a 32-bit word replaces the compiler's select of
// both words of a conditionally added alpha.
template<class Emit>
__device__ __forceinline__ void walk_loop_fast(const Grid& g, Walk& w, double& prev, bool active, Emit&& emit)
{
  double end = w.amax;
#pragma unroll
  for (int d = 0; d < 3; ++d)
  {
    const double x = w.left[d] > 0 ? dadd(w.a[d], dmul((double)w.left[d], w.da[d])) : w.a[d];
    const double lim = dsub(dsub(x, kEps), dmul(x, 0x1p-20));
    end = (lim < end || lim != lim) ? lim : end;  // a NaN bound leaves every step to the checked loop
  }
  if (active)
  {
    double big = 0.0;
    int da_hi[3], da_lo[3];
#pragma unroll
    for (int d = 0; d < 3; ++d)
    {
      big = (w.a[d] < 1.0 && w.da[d] > big) ? w.da[d] : big;
      da_hi[d] = __double2hiint(w.da[d]);
      da_lo[d] = __double2loint(w.da[d]);
    }
    const double end2 = dsub(dsub(end, big), 4.0 * kEps);
    // one unchecked step from prev (its minimum m is below end)
    auto step = [&](double m) {
      emit(true, w.c, dmul(dsub(m, prev), w.d12));
      const double thr = __dadd_ru(m, kEps);
#pragma unroll
      for (int d = 0; d < 3; ++d)
      {
        const bool p = w.a[d] < thr;
        w.a[d] = dadd(w.a[d], __hiloint2double(p ? da_hi[d] : 0, da_lo[d]));
        w.c += p ? w.step[d] : 0;
      }
      prev = m;
    };
    while (true)
    {
      const double m = min_of(w.a[0], min_of(w.a[1], w.a[2]));
      if (!(m < end2))
      {
        break;
      }
      step(m);
      step(min_of(w.a[0], min_of(w.a[1], w.a[2])));
    }
    while (true)
    {
      const double m = min_of(w.a[0], min_of(w.a[1], w.a[2]));
      if (!(m < end))
      {
        break;
      }
      step(m);
    }
    left_from_index(g, w);
  }
  bool more = active;
  while (more)
  {
    const double n1 = walk_step<true>(w, prev, more, emit);
    if (!more)
    {
      prev = n1;
      break;
    }
    prev = walk_step<true>(w, n1, more, emit);
  }
}

// The general form, bounded by the step guard (non-finite input can make a
// step advance nothing).
template<class Emit>
__device__ __forceinline__ void walk_loop_exact(Walk& w, double& prev, int& guard, bool active, Emit&& emit)
{
  bool more = active;
  while (more)
  {
    prev = walk_step<false>(w, prev, more, emit);
    --guard;
    more = more && guard > 0;
  }
}

// emit(inside, linearIndex, length) is called for every element FIR stores
// (inside is always true; the parameter keeps the emitters' form).  Lanes
// with nothing to trace pass go = false.  All lanes of the warp must call
// this together (it votes on the tie form); a kernel that traverses twice
// per lane calls __syncwarp() between the traversals.  Returns false for a
// lane that hit the step bound, which only non-finite input can cause.
template<class Emit>
__device__ __forceinline__ bool siddon_walk(const Grid& g, Walk w, bool go, Emit&& emit)
{
  double prev = w.amin;
  int guard = g.guard;
  const bool active = go && prev < w.amax;
  // every alpha of the walk is >= the smallest initial one (alphas only
  // grow, alphaMax > alphaMin), so this decides the tie form for the walk
  const bool fast =
    !active || (!g.exact_only && min_of(w.amin, min_of(w.a[0], min_of(w.a[1], w.a[2]))) >= kEps);
  if (__all_sync(__activemask(), fast))
  {
    walk_loop_fast(g, w, prev, active, emit);
  }
  else
  {
    walk_loop_exact(w, prev, guard, active, emit);
  }
  // stopped by the bound: still inside, before alphaMax
  return !go || !(prev < w.amax) || (w.left[0] | w.left[1] | w.left[2]) < 0;
}

// VolData::computeLineIntegral accumulation step (VolData.cc:362-368): the
// float running sum is widened, the double product added, the sum rounded.
// `value` is the voxel widened to double: the projectors gather from a
// double copy of the float image (exact), which saves a conversion per step.
__device__ __forceinline__ float accumulate(float line, double length, double value)
{
  return __double2float_rn(dadd((double)line, dmul(length, value)));
}

}  // namespace fir
