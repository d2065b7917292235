// Host-side formats around the path: the Gmsh MSH 2.2 surface reader of
// the marker initialisation, the restart file of read_restart /
// write_restart, and the Tecplot POINT dump of write_flowfield.  Plain
// C++ (no device code): a caller converting a real FEICAR case reads its
// surface and restart through these and hands the arrays to the case.
#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/feicar_b200.h"

namespace {

// ------------------------------------------------------------- MSH 2.2

struct LineReader {
  FILE *f;
  std::string line;
  long long lineno = 0;
  explicit LineReader(FILE *fp) : f(fp) {}
  bool next() {
    line.clear();
    int ch;
    bool any = false;
    while ((ch = fgetc(f)) != EOF) {
      any = true;
      if (ch == '\n') break;
      line.push_back((char)ch);
    }
    if (!any) return false;
    while (!line.empty() && (line.back() == '\r' || line.back() == ' ' || line.back() == '\t')) line.pop_back();
    ++lineno;
    return true;
  }
  // the first token of the line (section names)
  std::string head() const {
    size_t a = line.find_first_not_of(" \t");
    if (a == std::string::npos) return std::string();
    size_t b = line.find_first_of(" \t", a);
    return line.substr(a, b == std::string::npos ? std::string::npos : b - a);
  }
};

bool parse_ll(const char *&p, long long *v) {
  char *e = nullptr;
  errno = 0;
  const long long x = strtoll(p, &e, 10);
  if (e == p || errno) return false;
  *v = x;
  p = e;
  return true;
}

bool parse_d(const char *&p, double *v) {
  char *e = nullptr;
  errno = 0;
  const double x = strtod(p, &e);
  if (e == p) return false;
  *v = x;
  p = e;
  return true;
}

bool skip_to(LineReader &r, const char *end_tag) {
  while (r.next())
    if (r.head() == end_tag) return true;
  return false;
}

fg_status msh_fail(FILE *f, fg_status s) {
  if (f) fclose(f);
  return s;
}

// ------------------------------------------------------ restart records

long long g_max_subrecord = 2147483639LL;  // 2**31 - 9

// One record of an unformatted sequential file: 4-byte length markers
// around each subrecord; every subrecord but the last has a negative
// leading marker, every subrecord but the first a negative trailing one.
struct RecordWriter {
  FILE *f;
  std::vector<unsigned char> buf;
  void add(const void *p, size_t n) {
    const unsigned char *c = static_cast<const unsigned char *>(p);
    buf.insert(buf.end(), c, c + n);
  }
  void zeros(size_t n) { buf.insert(buf.end(), n, 0); }
  bool flush() {
    const size_t total = buf.size();
    size_t off = 0;
    bool first = true;
    do {
      const size_t len = std::min<size_t>(total - off, (size_t)g_max_subrecord);
      const bool last = off + len == total;
      const int32_t lead = last ? (int32_t)len : -(int32_t)len;
      const int32_t trail = first ? (int32_t)len : -(int32_t)len;
      if (fwrite(&lead, 4, 1, f) != 1) return false;
      if (len && fwrite(buf.data() + off, 1, len, f) != len) return false;
      if (fwrite(&trail, 4, 1, f) != 1) return false;
      off += len;
      first = false;
    } while (off < total);
    buf.clear();
    return true;
  }
};

bool read_record(FILE *f, std::vector<unsigned char> &out) {
  out.clear();
  for (;;) {
    int32_t lead, trail;
    if (fread(&lead, 4, 1, f) != 1) return false;
    const bool more = lead < 0;
    const long long len = more ? -(long long)lead : (long long)lead;
    const size_t at = out.size();
    out.resize(at + (size_t)len);
    if (len && fread(out.data() + at, 1, (size_t)len, f) != (size_t)len) return false;
    if (fread(&trail, 4, 1, f) != 1) return false;
    if ((trail < 0 ? -(long long)trail : (long long)trail) != len) return false;
    if (!more) return true;
  }
}

struct Piece {
  void *p;
  size_t bytes;
};

// the arrays of the flow record in write order (MAIN.F90:1082-1091)
std::vector<Piece> flow_pieces(const fg_restart_flow *f) {
  const size_t NX = (size_t)f->nx + 2, NY = (size_t)f->ny + 2, NZ = (size_t)f->nz + 2;
  const size_t n3 = NX * NY * NZ * sizeof(double);
  const size_t bx = 2 * NY * NZ * sizeof(double), by = NX * 2 * NZ * sizeof(double),
               bz = NX * NY * 2 * sizeof(double);
  const size_t gx = NY * NZ * sizeof(double), gy = NX * NZ * sizeof(double), gz = NX * NY * sizeof(double);
  std::vector<Piece> v = {
      {f->u, n3},    {f->v, n3},    {f->w, n3},    {f->p, n3},    {f->face_u, n3}, {f->face_v, n3},
      {f->face_w, n3}, {f->pPrime, n3},
      {f->bcxu, bx}, {f->bcxv, bx}, {f->bcxw, bx}, {f->bcxp, bx},
      {f->bcyu, by}, {f->bcyv, by}, {f->bcyw, by}, {f->bcyp, by},
      {f->bczu, bz}, {f->bczv, bz}, {f->bczw, bz}, {f->bczp, bz},
      {f->pgrad[0], gx}, {f->pgrad[1], gx}, {f->pgrad[2], gy}, {f->pgrad[3], gy}, {f->pgrad[4], gz},
      {f->pgrad[5], gz},
      {f->iblank, NX * NY * NZ}, {f->ghostcellmark, NX * NY * NZ}};
  return v;
}

// ------------------------------------------------------------ Tecplot

// Fortran 1PE12.5: d.dddddE+xx, or d.ddddd+xxx for a three-digit exponent
void put_pe12_5(std::string &s, double v) {
  char b[40];
  if (std::isnan(v)) {
    s.append("         NaN");
    return;
  }
  if (std::isinf(v)) {
    s.append(v > 0 ? "    Infinity" : "   -Infinity");
    return;
  }
  int n = snprintf(b, sizeof b, "%.5E", v);
  char *e = strchr(b, 'E');
  if (e && n > 0) {
    const int ex = atoi(e + 1);
    if (ex >= 100 || ex <= -100) {
      // drop the exponent letter: the sign and three digits follow the mantissa
      memmove(e, e + 1, strlen(e + 1) + 1);
      n = (int)strlen(b);
    }
  }
  for (int k = n; k < 12; ++k) s.push_back(' ');
  if (n > 12) {
    s.append(12, '*');
    return;
  }
  s.append(b, (size_t)n);
}

void put_i2(std::string &s, int v) {
  if (v > 99 || v < -9) {
    s.append("**");
    return;
  }
  char b[8];
  snprintf(b, sizeof b, "%2d", v);
  s.append(b);
}

}  // namespace

extern "C" {

fg_status fg_read_msh22(const char *path, int *nvert, int *ntri, double *xyz, int cap_vert, int *tri,
                        int cap_tri, int *nskipped) {
  if (!path || !nvert || !ntri) return FG_BAD_INPUT;
  FILE *f = fopen(path, "r");
  if (!f) return FG_IO_ERROR;
  LineReader r(f);
  bool have_nodes = false, have_elems = false;
  std::unordered_map<long long, int> tag_to_index;
  std::vector<double> nodes;
  std::vector<long long> elems;  // node tags, 3 per triangle
  long long skipped = 0;
  while (r.next()) {
    const std::string h = r.head();
    if (h == "$MeshFormat") {
      if (!r.next()) return msh_fail(f, FG_IO_ERROR);
      const char *p = r.line.c_str();
      double version;
      long long ftype;
      if (!parse_d(p, &version) || !parse_ll(p, &ftype)) return msh_fail(f, FG_IO_ERROR);
      if (version < 2.0 || version >= 3.0 || ftype != 0) return msh_fail(f, FG_IO_ERROR);  // ASCII 2.x only
      if (!skip_to(r, "$EndMeshFormat")) return msh_fail(f, FG_IO_ERROR);
    } else if (h == "$Nodes") {
      if (!r.next()) return msh_fail(f, FG_IO_ERROR);
      const char *p = r.line.c_str();
      long long n;
      if (!parse_ll(p, &n) || n < 0 || n > (1LL << 30)) return msh_fail(f, FG_IO_ERROR);
      nodes.resize(3 * (size_t)n);
      tag_to_index.reserve((size_t)n);
      for (long long q = 0; q < n; ++q) {
        if (!r.next()) return msh_fail(f, FG_IO_ERROR);
        const char *s = r.line.c_str();
        long long tag;
        if (!parse_ll(s, &tag) || !parse_d(s, &nodes[3 * q]) || !parse_d(s, &nodes[3 * q + 1]) ||
            !parse_d(s, &nodes[3 * q + 2]))
          return msh_fail(f, FG_IO_ERROR);
        tag_to_index[tag] = (int)q;
      }
      if (!r.next() || r.head() != "$EndNodes") return msh_fail(f, FG_IO_ERROR);
      have_nodes = true;
    } else if (h == "$Elements") {
      if (!r.next()) return msh_fail(f, FG_IO_ERROR);
      const char *p = r.line.c_str();
      long long n;
      if (!parse_ll(p, &n) || n < 0 || n > (1LL << 30)) return msh_fail(f, FG_IO_ERROR);
      elems.reserve(3 * (size_t)n);
      for (long long q = 0; q < n; ++q) {
        if (!r.next()) return msh_fail(f, FG_IO_ERROR);
        const char *s = r.line.c_str();
        long long num, type, ntags, t;
        if (!parse_ll(s, &num) || !parse_ll(s, &type) || !parse_ll(s, &ntags) || ntags < 0)
          return msh_fail(f, FG_IO_ERROR);
        for (long long k = 0; k < ntags; ++k)
          if (!parse_ll(s, &t)) return msh_fail(f, FG_IO_ERROR);
        if (type != 2) {  // only 3-node triangles make a body surface
          ++skipped;
          continue;
        }
        long long a, b, c;
        if (!parse_ll(s, &a) || !parse_ll(s, &b) || !parse_ll(s, &c)) return msh_fail(f, FG_IO_ERROR);
        elems.push_back(a);
        elems.push_back(b);
        elems.push_back(c);
      }
      if (!r.next() || r.head() != "$EndElements") return msh_fail(f, FG_IO_ERROR);
      have_elems = true;
    }
    // $PhysicalNames and any other section: read past (the physical tags
    // name the surface but do not enter the path)
  }
  fclose(f);
  if (!have_nodes || !have_elems) return FG_IO_ERROR;
  const long long nv = (long long)nodes.size() / 3, nt = (long long)elems.size() / 3;
  if (nv > 0x7fffffff || nt > 0x7fffffff) return FG_BAD_INPUT;
  *nvert = (int)nv;
  *ntri = (int)nt;
  if (nskipped) *nskipped = (int)skipped;
  if (!xyz && !tri) return FG_OK;
  if (!xyz || !tri || cap_vert < nv || cap_tri < nt) return FG_BAD_INPUT;
  memcpy(xyz, nodes.data(), nodes.size() * sizeof(double));
  for (size_t k = 0; k < elems.size(); ++k) {
    auto it = tag_to_index.find(elems[k]);
    if (it == tag_to_index.end()) return FG_BAD_INPUT;  // a triangle names a node that is not in $Nodes
    tri[k] = it->second;
  }
  return FG_OK;
}

void fg_set_max_subrecord(long long bytes) {
  g_max_subrecord = (bytes >= 16 && bytes <= 2147483639LL) ? bytes : 2147483639LL;
}

fg_status fg_write_restart(const char *path, const fg_restart_flow *fl, int nbody, const fg_restart_body *b) {
  if (!path || !fl || fl->nx < 1 || fl->ny < 1 || fl->nz < 1 || nbody < 0 || (nbody > 0 && !b))
    return FG_BAD_INPUT;
  FILE *f = fopen(path, "wb");
  if (!f) return FG_IO_ERROR;
  RecordWriter w{f, {}};
  bool ok = true;
  // time, ntime (MAIN.F90:1081)
  const double t = fl->time;
  const int32_t nt = (int32_t)fl->ntime;
  w.add(&t, 8);
  w.add(&nt, 4);
  ok = ok && w.flush();
  for (const Piece &pc : flow_pieces(fl)) {
    if (pc.p) w.add(pc.p, pc.bytes);
    else w.zeros(pc.bytes);
  }
  ok = ok && w.flush();
  // one record per body (MAIN.F90:1094-1110)
  for (int ib = 0; ok && ib < nbody; ++ib) {
    const fg_restart_body &B = b[ib];
    if (B.npts < 0 || B.nelm < 0) {
      fclose(f);
      return FG_BAD_INPUT;
    }
    const size_t nb = (size_t)B.npts * sizeof(double);
    for (const double *a : {B.x, B.y, B.z, B.u, B.v, B.w, B.fx, B.fy, B.fz}) {
      if (a) w.add(a, nb);
      else w.zeros(nb);
    }
    for (int e = 0; e < 3 * B.nelm; ++e) {
      const int32_t one_based = B.tri ? (int32_t)B.tri[e] + 1 : 0;  // triElemNeig is 1-based
      w.add(&one_based, 4);
    }
    for (const double *s : {B.cent, B.ang, B.vcent, B.angv}) w.add(s, 3 * sizeof(double));
    ok = w.flush();
  }
  if (fclose(f) != 0) ok = false;
  return ok ? FG_OK : FG_IO_ERROR;
}

fg_status fg_read_restart(const char *path, fg_restart_flow *fl, int nbody, fg_restart_body *b) {
  if (!path || !fl || fl->nx < 1 || fl->ny < 1 || fl->nz < 1 || nbody < 0 || (nbody > 0 && !b))
    return FG_BAD_INPUT;
  FILE *f = fopen(path, "rb");
  if (!f) return FG_IO_ERROR;
  std::vector<unsigned char> rec;
  // time, ntime_start (MAIN.F90:1008)
  if (!read_record(f, rec) || rec.size() != 12) {
    fclose(f);
    return FG_IO_ERROR;
  }
  int32_t nt;
  memcpy(&fl->time, rec.data(), 8);
  memcpy(&nt, rec.data() + 8, 4);
  fl->ntime = nt;
  const std::vector<Piece> pcs = flow_pieces(fl);
  size_t need = 0;
  for (const Piece &pc : pcs) need += pc.bytes;
  if (!read_record(f, rec) || rec.size() != need) {
    fclose(f);
    return FG_IO_ERROR;
  }
  size_t off = 0;
  for (const Piece &pc : pcs) {
    if (pc.p) memcpy(pc.p, rec.data() + off, pc.bytes);
    off += pc.bytes;
  }
  for (int ib = 0; ib < nbody; ++ib) {
    fg_restart_body &B = b[ib];
    const size_t nb = (size_t)B.npts * sizeof(double);
    if (B.npts < 0 || B.nelm < 0 || !read_record(f, rec) ||
        rec.size() != 9 * nb + 12 * (size_t)B.nelm + 12 * sizeof(double)) {
      fclose(f);
      return FG_IO_ERROR;
    }
    off = 0;
    for (double *a : {B.x, B.y, B.z, B.u, B.v, B.w, B.fx, B.fy, B.fz}) {
      if (a) memcpy(a, rec.data() + off, nb);
      off += nb;
    }
    for (int e = 0; e < 3 * B.nelm; ++e) {
      int32_t v;
      memcpy(&v, rec.data() + off, 4);
      off += 4;
      if (B.tri) B.tri[e] = v - 1;
    }
    for (double *s : {B.cent, B.ang, B.vcent, B.angv}) {
      memcpy(s, rec.data() + off, 3 * sizeof(double));
      off += 3 * sizeof(double);
    }
  }
  fclose(f);
  return FG_OK;
}

fg_status fg_write_tecplot(const char *path, int nx, int ny, int nz, const double *xc, const double *yc,
                           const double *zc, const fg_tecplot_fields *fd) {
  if (!path || nx < 1 || ny < 1 || nz < 1 || !xc || !yc || !zc) return FG_BAD_INPUT;
  fg_tecplot_fields z{};
  const fg_tecplot_fields &F = fd ? *fd : z;
  FILE *f = fopen(path, "w");
  if (!f) return FG_IO_ERROR;
  bool ok = true;
  // write_flowfield, nDim = 3 (UTIL_GENERAL.F90:200-219)
  ok = ok && fputs("VARIABLES=\"X\",\"Y\",\"Z\",\"U\",\"V\",\"W\",\"P\",\"OX\",\"OY\",\"OZ\",\"LMD\",\"IBLANK\","
                   "\"GHOST\",\"DEAD\",\"B#\",\"goa\"\n", f) >= 0;
  ok = ok && fprintf(f, " ZONE F=POINT, I=%d, J=%d K=%d\n", nx + 1, ny + 1, nz + 1) > 0;
  const size_t NX = (size_t)nx + 2, NY = (size_t)ny + 2;
  const double *re[8] = {F.u, F.v, F.w, F.p, F.ox, F.oy, F.oz, F.lmd};
  const int8_t *in[5] = {F.iblank, F.ghost, F.dead, F.bodynum, F.goa};
  std::vector<std::string> planes((size_t)nz + 1);
  // planes formatted in parallel, written in order
  const int chunk = 16;
  for (int k0 = 0; ok && k0 <= nz; k0 += chunk) {
    const int k1 = std::min(nz, k0 + chunk - 1);
#pragma omp parallel for schedule(dynamic, 1)
    for (int k = k0; k <= k1; ++k) {
      std::string &s = planes[(size_t)k];
      s.clear();
      s.reserve((size_t)(nx + 1) * (ny + 1) * 170);
      for (int j = 0; j <= ny; ++j)
        for (int i = 0; i <= nx; ++i) {
          const size_t id = (size_t)i + NX * ((size_t)j + NY * (size_t)k);
          const double c3[3] = {xc[i], yc[j], zc[k]};
          for (double v : c3) {
            s.append("  ");
            put_pe12_5(s, v);
          }
          for (const double *a : re) {
            s.append("  ");
            put_pe12_5(s, a ? a[id] : 0.0);
          }
          for (const int8_t *a : in) {
            s.append("  ");
            put_i2(s, a ? (int)a[id] : 0);
          }
          s.push_back('\n');
        }
    }
    for (int k = k0; ok && k <= k1; ++k) {
      std::string &s = planes[(size_t)k];
      ok = fwrite(s.data(), 1, s.size(), f) == s.size();
      std::string().swap(s);
    }
  }
  if (fclose(f) != 0) ok = false;
  return ok ? FG_OK : FG_IO_ERROR;
}

}  // extern "C"
