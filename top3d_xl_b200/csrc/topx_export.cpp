// Design output files (TOP3D_XL.m:206-222, 564-577): the padded density volume as NIfTI-1 and its
// 0.5 isosurface, closed by caps on the volume boundary, as binary STL.
//
// The reference flips the volume along y, applies smooth3(V, 'box', 1) (a box of size 1, which
// leaves it unchanged), and takes isosurface(V, 0.5) plus isocaps(V, 0.5) with MATLAB's
// vertex coordinates: x = column, y = row, z = page, samples at 1-based integer positions.
// The surface here is extracted by marching tetrahedra: every lattice cube is cut into six
// tetrahedra around its main diagonal, a cut whose face diagonals agree between neighbouring
// cubes, so the surface has no cracks.  The caps cut each boundary square along the same
// diagonals and fill the part of each triangle whose values lie above the isovalue.  Every
// crossing point is computed from its two lattice samples in one fixed order, so surface and
// caps share vertices exactly and the triangle set is closed.  Triangles face away from the
// region above the isovalue.  The triangulation differs from MATLAB's marching cubes; the
// isovalue, orientation, coordinates and closure follow the reference.
#include <array>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "topx.h"

namespace {

struct V3 {
  double x, y, z;
};
V3 sub(const V3& a, const V3& b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
V3 cross(const V3& a, const V3& b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
double dot(const V3& a, const V3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

// the flipped lattice: sample (i, j, k) = V(ny - 1 - i, j, k), at MATLAB position (j+1, i+1, k+1)
struct Lattice {
  const double* v;
  int ny, nx, nz;
  double iso;
  int64_t id(int i, int j, int k) const { return i + int64_t(ny) * (j + int64_t(nx) * k); }
  double val(int i, int j, int k) const { return v[(ny - 1 - i) + int64_t(ny) * (j + int64_t(nx) * k)]; }
  V3 pos(int i, int j, int k) const { return {double(j + 1), double(i + 1), double(k + 1)}; }
};

struct Pt {
  int i, j, k;
};

class Mesh {
 public:
  explicit Mesh(const Lattice& L) : L_(L) {}
  std::vector<std::array<V3, 3>> tris;

  // crossing of the isovalue on edge a-b, from the endpoints in lattice-index order
  V3 cross_point(const Pt& a, const Pt& b) const {
    const bool swap = L_.id(b.i, b.j, b.k) < L_.id(a.i, a.j, a.k);
    const Pt& p = swap ? b : a;
    const Pt& q = swap ? a : b;
    const double vp = L_.val(p.i, p.j, p.k), vq = L_.val(q.i, q.j, q.k);
    const double t = (L_.iso - vp) / (vq - vp);
    const V3 P = L_.pos(p.i, p.j, p.k), Q = L_.pos(q.i, q.j, q.k);
    return {P.x + t * (Q.x - P.x), P.y + t * (Q.y - P.y), P.z + t * (Q.z - P.z)};
  }
  bool above(const Pt& a) const { return L_.val(a.i, a.j, a.k) > L_.iso; }
  V3 pos(const Pt& a) const { return L_.pos(a.i, a.j, a.k); }

  // add triangle (p0, p1, p2) with its normal along `out` (skipped when degenerate)
  void add(V3 p0, V3 p1, V3 p2, const V3& out) {
    const V3 n = cross(sub(p1, p0), sub(p2, p0));
    const double d = dot(n, out);
    if (d == 0.0 || !std::isfinite(d)) return;
    if (d < 0) std::swap(p1, p2);
    tris.push_back({p0, p1, p2});
  }

  // surface piece inside tetrahedron t[0..3]
  void tet(const Pt (&t)[4]) {
    int in[4], out[4], ni = 0, no = 0;
    for (int a = 0; a < 4; ++a) (above(t[a]) ? in[ni++] : out[no++]) = a;
    if (ni == 0 || no == 0) return;
    V3 ci{0, 0, 0}, co{0, 0, 0};
    for (int a = 0; a < ni; ++a) ci = {ci.x + pos(t[in[a]]).x, ci.y + pos(t[in[a]]).y, ci.z + pos(t[in[a]]).z};
    for (int a = 0; a < no; ++a) co = {co.x + pos(t[out[a]]).x, co.y + pos(t[out[a]]).y, co.z + pos(t[out[a]]).z};
    const V3 dir = sub({co.x / no, co.y / no, co.z / no}, {ci.x / ni, ci.y / ni, ci.z / ni});
    if (ni == 1 || no == 1) {  // one vertex alone on its side: one triangle
      const int s = ni == 1 ? in[0] : out[0];
      V3 q[3];
      for (int a = 0, m = 0; a < 4; ++a)
        if (a != s) q[m++] = cross_point(t[s], t[a]);
      add(q[0], q[1], q[2], dir);
    } else {  // two and two: a quadrilateral
      const Pt &a = t[in[0]], &b = t[in[1]], &c = t[out[0]], &d = t[out[1]];
      const V3 ac = cross_point(a, c), ad = cross_point(a, d), bd = cross_point(b, d), bc = cross_point(b, c);
      add(ac, ad, bd, dir);
      add(ac, bd, bc, dir);
    }
  }

  // cap piece of boundary triangle (a, b, c) whose outward normal is `out`
  void cap(const Pt& a, const Pt& b, const Pt& c, const V3& out) {
    const Pt t[3] = {a, b, c};
    int in[3], ou[3], ni = 0, no = 0;
    for (int m = 0; m < 3; ++m) (above(t[m]) ? in[ni++] : ou[no++]) = m;
    if (ni == 0) return;
    if (ni == 3) {
      add(pos(a), pos(b), pos(c), out);
    } else if (ni == 2) {
      const Pt &p = t[in[0]], &q = t[in[1]], &r = t[ou[0]];
      const V3 qr = cross_point(q, r), pr = cross_point(p, r);
      add(pos(p), pos(q), qr, out);
      add(pos(p), qr, pr, out);
    } else {
      const Pt &p = t[in[0]], &q = t[ou[0]], &r = t[ou[1]];
      add(pos(p), cross_point(p, q), cross_point(p, r), out);
    }
  }

 private:
  const Lattice& L_;
};

// cube corners in (x, y, z) = (j, i, k) offsets
constexpr int kCorner[8][3] = {{0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0}, {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
// six tetrahedra around the diagonal 0-6
constexpr int kTet[6][4] = {{0, 1, 2, 6}, {0, 2, 3, 6}, {0, 3, 7, 6}, {0, 7, 4, 6}, {0, 4, 5, 6}, {0, 5, 1, 6}};

Pt corner(int i, int j, int k, int c) { return {i + kCorner[c][1], j + kCorner[c][0], k + kCorner[c][2]}; }

}  // namespace

extern "C" {

topx_status topx_write_design_stl(const double* vol, int ny, int nx, int nz, double iso, const char* path,
                                  int64_t* ntriangles) {
  if (!vol || !path || ny < 2 || nx < 2 || nz < 2 || !std::isfinite(iso)) return TOPX_ERR_ARG;
  try {
    const Lattice L{vol, ny, nx, nz, iso};
    Mesh M(L);
    for (int k = 0; k + 1 < nz; ++k)
      for (int j = 0; j + 1 < nx; ++j)
        for (int i = 0; i + 1 < ny; ++i)
          for (const auto& tt : kTet) {
            const Pt t[4] = {corner(i, j, k, tt[0]), corner(i, j, k, tt[1]), corner(i, j, k, tt[2]),
                             corner(i, j, k, tt[3])};
            M.tet(t);
          }
    // caps: boundary squares cut along the tetrahedra's face diagonals
    auto face = [&](int i, int j, int k, int a, int b, int c, const V3& out) {
      M.cap(corner(i, j, k, a), corner(i, j, k, b), corner(i, j, k, c), out);
    };
    for (int k = 0; k + 1 < nz; ++k)
      for (int i = 0; i + 1 < ny; ++i) {
        face(i, 0, k, 0, 3, 7, {-1, 0, 0});  // x = 1
        face(i, 0, k, 0, 7, 4, {-1, 0, 0});
        face(i, nx - 2, k, 1, 2, 6, {1, 0, 0});  // x = nx
        face(i, nx - 2, k, 1, 6, 5, {1, 0, 0});
      }
    for (int k = 0; k + 1 < nz; ++k)
      for (int j = 0; j + 1 < nx; ++j) {
        face(0, j, k, 0, 4, 5, {0, -1, 0});  // y = 1
        face(0, j, k, 0, 5, 1, {0, -1, 0});
        face(ny - 2, j, k, 2, 3, 6, {0, 1, 0});  // y = ny
        face(ny - 2, j, k, 3, 7, 6, {0, 1, 0});
      }
    for (int j = 0; j + 1 < nx; ++j)
      for (int i = 0; i + 1 < ny; ++i) {
        face(i, j, 0, 0, 1, 2, {0, 0, -1});  // z = 1
        face(i, j, 0, 0, 2, 3, {0, 0, -1});
        face(i, j, nz - 2, 7, 4, 6, {0, 0, 1});  // z = nz
        face(i, j, nz - 2, 4, 5, 6, {0, 0, 1});
      }
    if (M.tris.size() > 0xffffffffu) return TOPX_ERR_ARG;
    FILE* f = std::fopen(path, "wb");
    if (!f) return TOPX_ERR_ARG;
    char header[80] = {};
    std::snprintf(header, sizeof(header), "topx DesignVolume isosurface %.6g with caps", iso);
    const uint32_t n = uint32_t(M.tris.size());
    bool ok = std::fwrite(header, 1, 80, f) == 80 && std::fwrite(&n, 4, 1, f) == 1;
    for (const auto& t : M.tris) {
      if (!ok) break;
      V3 nn = cross(sub(t[1], t[0]), sub(t[2], t[0]));
      const double len = std::sqrt(dot(nn, nn));
      float rec[12] = {float(nn.x / len), float(nn.y / len), float(nn.z / len)};
      for (int m = 0; m < 3; ++m) {
        rec[3 + 3 * m] = float(t[m].x);
        rec[4 + 3 * m] = float(t[m].y);
        rec[5 + 3 * m] = float(t[m].z);
      }
      const uint16_t attr = 0;
      ok = std::fwrite(rec, 4, 12, f) == 12 && std::fwrite(&attr, 2, 1, f) == 1;
    }
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) return TOPX_ERR_ARG;
    if (ntriangles) *ntriangles = int64_t(n);
    return TOPX_OK;
  } catch (...) {
    return TOPX_ERR_INTERNAL;
  }
}

// NIfTI-1 single file: 348-byte header, 4-byte extension flag, then the volume (FLOAT64, first
// index fastest, as V(y, x, z) is stored) -- what niftiwrite(V, fileName) writes (TX:564-570).
#pragma pack(push, 1)
struct Nifti1Header {
  int32_t sizeof_hdr;
  char data_type[10], db_name[18];
  int32_t extents;
  int16_t session_error;
  char regular, dim_info;
  int16_t dim[8];
  float intent_p1, intent_p2, intent_p3;
  int16_t intent_code, datatype, bitpix, slice_start;
  float pixdim[8];
  float vox_offset, scl_slope, scl_inter;
  int16_t slice_end;
  char slice_code, xyzt_units;
  float cal_max, cal_min, slice_duration, toffset;
  int32_t glmax, glmin;
  char descrip[80], aux_file[24];
  int16_t qform_code, sform_code;
  float quatern_b, quatern_c, quatern_d, qoffset_x, qoffset_y, qoffset_z;
  float srow_x[4], srow_y[4], srow_z[4];
  char intent_name[16], magic[4];
};
#pragma pack(pop)
static_assert(sizeof(Nifti1Header) == 348, "NIfTI-1 header size");

topx_status topx_write_design_nii(const double* vol, int ny, int nx, int nz, const char* path) {
  if (!vol || !path || ny < 1 || nx < 1 || nz < 1 || ny > 32767 || nx > 32767 || nz > 32767) return TOPX_ERR_ARG;
  Nifti1Header h;
  std::memset(&h, 0, sizeof(h));
  h.sizeof_hdr = 348;
  h.regular = 'r';
  h.dim[0] = 3;
  h.dim[1] = int16_t(ny);
  h.dim[2] = int16_t(nx);
  h.dim[3] = int16_t(nz);
  for (int d = 4; d < 8; ++d) h.dim[d] = 1;
  h.datatype = 64;  // DT_FLOAT64
  h.bitpix = 64;
  for (int d = 0; d < 8; ++d) h.pixdim[d] = 1.0f;  // pixdim[0] = qfac
  h.vox_offset = 352.0f;
  h.scl_slope = 1.0f;
  h.xyzt_units = 2;  // millimetres, as niftiwrite's default header
  h.srow_x[0] = h.srow_y[1] = h.srow_z[2] = 1.0f;
  std::snprintf(h.descrip, sizeof(h.descrip), "topx DesignVolume");
  std::memcpy(h.magic, "n+1", 4);
  FILE* f = std::fopen(path, "wb");
  if (!f) return TOPX_ERR_ARG;
  const char ext[4] = {0, 0, 0, 0};
  const size_t n = size_t(ny) * nx * nz;
  bool ok = std::fwrite(&h, sizeof(h), 1, f) == 1 && std::fwrite(ext, 1, 4, f) == 4 &&
            std::fwrite(vol, sizeof(double), n, f) == n;
  ok = (std::fclose(f) == 0) && ok;
  return ok ? TOPX_OK : TOPX_ERR_ARG;
}

}  // extern "C"
