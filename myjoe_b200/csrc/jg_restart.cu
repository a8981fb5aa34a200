// The reference's binary restart file, read and written on the host, and the
// bridge between such a file and a case handle's device state.
//
// Format (Ugp.cpp:9792-9820 ids, 9822-9898 header type, 9902-10660 writer,
// 12473-12800 reader; Ugp.h:3423-3446 header): two ints (magic 123581321,
// version 1), then 256-byte headers {char name[52]; int id; int64 skip;
// int idata[16]; double rdata[16]}, each followed by its payload; `skip` is
// the header plus payload size.  Order as Ugp::writeRestart lays it out with
// one process: counts, NO_CHECK, FA_CHECK, CV_CHECK, NOOFA_I_AND_V, CVOFA,
// one FA_ZONE header per face zone, CV_PART, X_NO, DATA, the data records
// (I0, D0, the D1 arrays, the D3 arrays, the D33 arrays, each class in the
// order it was registered), EOF.  Node, face and cell payloads are in global
// index order, which the check records state as 0..n-1.  A file written on
// a machine of the other byte order is recognised by its swapped magic
// number and swapped on reading (Ugp.cpp:10843-10853); files are written in
// the native order.
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/joe_b200.h"
#include "jg_internal.h"

namespace {

constexpr int kMagic = 123581321;
constexpr int kVersion = 1;
constexpr int kHeader = 256;
constexpr int kNameLen = 52;

enum {
  ID_COUNTS = 10, ID_I0 = 11, ID_D0 = 12,
  ID_FA_CHECK = 20, ID_NOOFA = 21, ID_CVOFA = 22, ID_FA_ZONE = 23, ID_FA_D1 = 24, ID_FA_D3 = 25,
  ID_NO_CHECK = 30, ID_X_NO = 31, ID_NO_D1 = 32, ID_NO_D3 = 33,
  ID_CV_CHECK = 40, ID_CV_PART = 41, ID_CV_D1 = 42, ID_CV_D3 = 43, ID_CV_D33 = 44,
  ID_DATA = 50, ID_EOF = 51
};

struct Header {
  char name[kNameLen];
  int32_t id;
  int64_t skip;
  int32_t idata[16];
  double rdata[16];
};
static_assert(sizeof(Header) == kHeader, "restart header must be 256 bytes");

struct Zone {
  std::string name;
  int kind = 0, ifa_f = 0, ifa_l = -1;
  double periodic[3] = {0.0, 0.0, 0.0};
};

struct Record {
  std::string name;
  int kind = 0;         // the UGP_IO_* id
  int count = 0;        // items (nodes, faces or cells); 0 for I0 / D0
  int width = 0;        // doubles per item: 1, 3 or 9
  int ivalue = 0;
  double dvalue = 0.0;
  std::vector<double> data;
};

int set_err(int code, const std::string& msg) { return jg::serve_set_err(code, msg.c_str()); }

int set_err(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  return jg::serve_set_err(code, buf);
}

int kind_width(int kind) {
  switch (kind) {
    case ID_I0: case ID_D0: return 0;
    case ID_FA_D1: case ID_NO_D1: case ID_CV_D1: return 1;
    case ID_FA_D3: case ID_NO_D3: case ID_CV_D3: return 3;
    case ID_CV_D33: return 9;
    default: return -1;
  }
}

// the class rank of a data record in the file: I0, D0, D1, D3, D33 (Ugp.cpp:10553-10625)
int kind_class(int kind) {
  switch (kind) {
    case ID_I0: return 0;
    case ID_D0: return 1;
    case ID_FA_D1: case ID_NO_D1: case ID_CV_D1: return 2;
    case ID_FA_D3: case ID_NO_D3: case ID_CV_D3: return 3;
    default: return 4;
  }
}

void swap4(void* p, size_t n) {
  auto* b = static_cast<unsigned char*>(p);
  for (size_t i = 0; i < n; i++, b += 4) {
    std::swap(b[0], b[3]);
    std::swap(b[1], b[2]);
  }
}

void swap8(void* p, size_t n) {
  auto* b = static_cast<unsigned char*>(p);
  for (size_t i = 0; i < n; i++, b += 8) {
    std::swap(b[0], b[7]);
    std::swap(b[1], b[6]);
    std::swap(b[2], b[5]);
    std::swap(b[3], b[4]);
  }
}

void swap_header(Header& h) {
  swap4(&h.id, 1);
  swap8(&h.skip, 1);
  swap4(h.idata, 16);
  swap8(h.rdata, 16);
}

Header make_header(const char* name, int id, int64_t skip) {
  Header h;
  std::memset(&h, 0, sizeof(h));
  std::strncpy(h.name, name, kNameLen - 1);
  h.id = id;
  h.skip = skip;
  return h;
}

std::string header_name(const Header& h) {
  return std::string(h.name, strnlen(h.name, kNameLen));
}

}  // namespace

struct jg_restart {
  bool has_mesh = false;
  int nno = 0, nfa = 0, ncv = 0, noofa_count = 0, nparts = 1;
  std::vector<double> x_no;      // [nno][3]
  std::vector<int> noofa_i;      // [nfa+1]
  std::vector<int> noofa_v;      // [noofa_count]
  std::vector<int> cvofa;        // [nfa][2]
  std::vector<int> cv_part;      // [ncv]
  std::vector<Zone> zones;
  std::vector<Record> records;

  int find(const char* name) const {
    for (size_t i = 0; i < records.size(); i++)
      if (records[i].name == name) return (int)i;
    return -1;
  }
};

namespace {

// a bounded cursor over the file's bytes
struct Reader {
  const std::vector<unsigned char>& buf;
  bool swap;
  int64_t pos = 0;
  bool take(void* dst, int64_t bytes) {
    if (bytes < 0 || pos + bytes > (int64_t)buf.size()) return false;
    std::memcpy(dst, buf.data() + pos, (size_t)bytes);
    pos += bytes;
    return true;
  }
  bool ints(int* dst, int64_t n) {
    if (!take(dst, 4 * n)) return false;
    if (swap) swap4(dst, (size_t)n);
    return true;
  }
  bool doubles(double* dst, int64_t n) {
    if (!take(dst, 8 * n)) return false;
    if (swap) swap8(dst, (size_t)n);
    return true;
  }
};

int check_index(const std::vector<int>& v, int n, const char* what) {
  for (size_t i = 0; i < v.size(); i++)
    if (v[i] != (int)i) return set_err(JG_ERR_IO, std::string("restart ") + what + " is not 0..n-1");
  (void)n;
  return JG_OK;
}

int parse(const std::vector<unsigned char>& buf, jg_restart& r) {
  Reader rd{buf, false};
  int magic[2];
  if (!rd.take(magic, 8)) return set_err(JG_ERR_IO, "restart file shorter than its magic number");
  if (magic[0] != kMagic) {
    swap4(magic, 2);
    if (magic[0] != kMagic) return set_err(JG_ERR_IO, "not a restart file (magic number)");
    rd.swap = true;
  }
  if (magic[1] != kVersion) return set_err(JG_ERR_IO, "restart io version " + std::to_string(magic[1]) + " (1 expected)");
  bool counts = false;
  int ndata_zone = 0;
  for (;;) {
    const int64_t at = rd.pos;
    Header h;
    if (!rd.take(&h, kHeader)) return set_err(JG_ERR_IO, "restart file ends before its EOF record");
    if (rd.swap) swap_header(h);
    if (h.skip < kHeader || at + h.skip > (int64_t)buf.size())
      return set_err(JG_ERR_IO, "restart record '" + header_name(h) + "' runs past the end of the file");
    const int id = h.id;
    if (id != ID_COUNTS && id != ID_EOF && !counts)
      return set_err(JG_ERR_IO, "restart record before the counts record");
    auto bad = [&](const char* why) {
      return set_err(JG_ERR_IO, "restart record '" + header_name(h) + "': " + why);
    };
    switch (id) {
      case ID_COUNTS:
        r.nno = h.idata[0];
        r.nfa = h.idata[1];
        r.ncv = h.idata[2];
        r.noofa_count = h.idata[3];
        if (r.nno < 0 || r.nfa < 0 || r.ncv < 0 || r.noofa_count < 0) return bad("negative count");
        counts = true;
        r.has_mesh = true;
        break;
      case ID_NO_CHECK:
      case ID_FA_CHECK:
      case ID_CV_CHECK: {
        const int n = id == ID_NO_CHECK ? r.nno : id == ID_FA_CHECK ? r.nfa : r.ncv;
        if (h.idata[0] != n || h.skip != kHeader + 4LL * n) return bad("size");
        std::vector<int> v((size_t)n);
        if (!rd.ints(v.data(), n)) return bad("truncated");
        int rc = check_index(v, n, header_name(h).c_str());
        if (rc) return rc;
        break;
      }
      case ID_NOOFA: {
        if (h.idata[0] != r.nfa || h.idata[1] != r.noofa_count ||
            h.skip != kHeader + 4LL * r.nfa + 4LL * r.noofa_count)
          return bad("size");
        std::vector<int> cnt((size_t)r.nfa);
        r.noofa_v.resize((size_t)r.noofa_count);
        if (!rd.ints(cnt.data(), r.nfa) || !rd.ints(r.noofa_v.data(), r.noofa_count)) return bad("truncated");
        r.noofa_i.assign((size_t)r.nfa + 1, 0);
        for (int f = 0; f < r.nfa; f++) {
          if (cnt[f] < 0) return bad("negative node count");
          r.noofa_i[f + 1] = r.noofa_i[f] + cnt[f];
        }
        if (r.noofa_i[r.nfa] != r.noofa_count) return bad("node counts do not add up");
        for (int v : r.noofa_v)
          if (v < 0 || v >= r.nno) return bad("node index out of range");
        break;
      }
      case ID_CVOFA:
        if (h.idata[0] != r.nfa || h.idata[1] != 2 || h.skip != kHeader + 8LL * r.nfa) return bad("size");
        r.cvofa.resize(2 * (size_t)r.nfa);
        if (!rd.ints(r.cvofa.data(), 2LL * r.nfa)) return bad("truncated");
        for (int f = 0; f < r.nfa; f++)
          if (r.cvofa[2 * f] < 0 || r.cvofa[2 * f] >= r.ncv || r.cvofa[2 * f + 1] >= r.ncv)
            return bad("cell index out of range");
        break;
      case ID_FA_ZONE: {
        if (h.skip != kHeader) return bad("size");
        Zone z;
        z.name = header_name(h);
        z.kind = h.idata[0];
        z.ifa_f = h.idata[1];
        z.ifa_l = h.idata[2];
        for (int k = 0; k < 3; k++) z.periodic[k] = h.rdata[k];
        if (z.ifa_f != ndata_zone || z.ifa_l < z.ifa_f - 1 || z.ifa_l >= r.nfa) return bad("face range");
        ndata_zone = z.ifa_l + 1;
        r.zones.push_back(z);
        break;
      }
      case ID_CV_PART:
        if (h.idata[0] != r.ncv || h.skip != kHeader + 4LL * r.ncv) return bad("size");
        r.nparts = h.idata[1];
        r.cv_part.resize((size_t)r.ncv);
        if (!rd.ints(r.cv_part.data(), r.ncv)) return bad("truncated");
        break;
      case ID_X_NO:
        if (h.idata[0] != r.nno || h.idata[1] != 3 || h.skip != kHeader + 24LL * r.nno) return bad("size");
        r.x_no.resize(3 * (size_t)r.nno);
        if (!rd.doubles(r.x_no.data(), 3LL * r.nno)) return bad("truncated");
        break;
      case ID_DATA:
        if (h.skip != kHeader) return bad("size");
        break;
      case ID_EOF:
        if (!counts) return set_err(JG_ERR_IO, "restart file without a counts record");
        if (ndata_zone != r.nfa) return set_err(JG_ERR_IO, "restart face zones do not cover every face");
        if (r.cvofa.empty() && r.nfa) return set_err(JG_ERR_IO, "restart file without CVOFA");
        if (r.noofa_i.empty()) r.noofa_i.assign((size_t)r.nfa + 1, 0);
        if (r.x_no.size() != 3 * (size_t)r.nno) return set_err(JG_ERR_IO, "restart file without X_NO");
        if (r.cv_part.empty()) r.cv_part.assign((size_t)r.ncv, 0);
        return JG_OK;
      default: {
        const int w = kind_width(id);
        if (w < 0) return bad("unknown record id");
        Record rec;
        rec.name = header_name(h);
        rec.kind = id;
        rec.width = w;
        if (id == ID_I0) {
          rec.ivalue = h.idata[0];
          if (h.skip != kHeader) return bad("size");
        } else if (id == ID_D0) {
          rec.dvalue = h.rdata[0];
          if (h.skip != kHeader) return bad("size");
        } else {
          const int n = (id == ID_FA_D1 || id == ID_FA_D3) ? r.nfa : (id == ID_NO_D1 || id == ID_NO_D3) ? r.nno : r.ncv;
          if (h.idata[0] != n || h.skip != kHeader + 8LL * n * w) return bad("size");
          if (w == 3 && h.idata[1] != 3) return bad("width");
          if (w == 9 && (h.idata[1] != 3 || h.idata[2] != 3)) return bad("width");
          rec.count = n;
          rec.data.resize((size_t)n * w);
          if (!rd.doubles(rec.data.data(), (int64_t)n * w)) return bad("truncated");
        }
        r.records.push_back(std::move(rec));
        break;
      }
    }
    rd.pos = at + h.skip;
  }
}

// appends bytes to the output image
struct Writer {
  std::vector<unsigned char> out;
  void put(const void* p, size_t bytes) {
    const auto* b = static_cast<const unsigned char*>(p);
    out.insert(out.end(), b, b + bytes);
  }
  void header(const Header& h) { put(&h, sizeof(h)); }
  void index_record(const char* name, int id, int n) {
    Header h = make_header(name, id, kHeader + 4LL * n);
    h.idata[0] = n;
    header(h);
    std::vector<int> v((size_t)n);
    for (int i = 0; i < n; i++) v[i] = i;
    put(v.data(), 4 * (size_t)n);
  }
};

int validate_mesh(const jg_restart& r) {
  if (!r.has_mesh) return set_err(JG_ERR_ARG, "restart has no mesh (jg_restart_set_mesh)");
  int next = 0;
  for (const Zone& z : r.zones) {
    if (z.ifa_f != next || z.ifa_l < z.ifa_f - 1) return set_err(JG_ERR_ARG, "face zones must be contiguous and in face order");
    next = z.ifa_l + 1;
  }
  if (next != r.nfa) return set_err(JG_ERR_ARG, "face zones must cover every face");
  return JG_OK;
}

}  // namespace

extern "C" {

int jg_restart_new(jg_restart_t** out) {
  if (!out) return set_err(JG_ERR_ARG, "null argument");
  *out = new jg_restart();
  return JG_OK;
}

int jg_restart_free(jg_restart_t* r) {
  delete r;
  return JG_OK;
}

int jg_restart_read(const char* path, jg_restart_t** out) {
  if (!path || !out) return set_err(JG_ERR_ARG, "null argument");
  *out = nullptr;
  FILE* f = std::fopen(path, "rb");
  if (!f) return set_err(JG_ERR_IO, std::string("cannot open restart file ") + path);
  std::vector<unsigned char> buf;
  unsigned char chunk[1 << 16];
  size_t n;
  while ((n = std::fread(chunk, 1, sizeof(chunk), f)) > 0) buf.insert(buf.end(), chunk, chunk + n);
  const bool err = std::ferror(f) != 0;
  std::fclose(f);
  if (err) return set_err(JG_ERR_IO, std::string("cannot read restart file ") + path);
  auto* r = new jg_restart();
  int rc = parse(buf, *r);
  if (rc) {
    delete r;
    return rc;
  }
  *out = r;
  return JG_OK;
}

int jg_restart_write(const jg_restart_t* r, const char* path) {
  if (!r || !path) return set_err(JG_ERR_ARG, "null argument");
  int rc = validate_mesh(*r);
  if (rc) return rc;
  Writer w;
  const int hdr_magic[2] = {kMagic, kVersion};
  w.put(hdr_magic, sizeof(hdr_magic));
  Header h = make_header("NO_FA_CV_NOOFA_COUNTS", ID_COUNTS, kHeader);
  h.idata[0] = r->nno;
  h.idata[1] = r->nfa;
  h.idata[2] = r->ncv;
  h.idata[3] = r->noofa_count;
  w.header(h);
  w.index_record("NO_CHECK", ID_NO_CHECK, r->nno);
  w.index_record("FA_CHECK", ID_FA_CHECK, r->nfa);
  w.index_record("CV_CHECK", ID_CV_CHECK, r->ncv);
  h = make_header("NOOFA_I_AND_V", ID_NOOFA, kHeader + 4LL * r->nfa + 4LL * r->noofa_count);
  h.idata[0] = r->nfa;
  h.idata[1] = r->noofa_count;
  w.header(h);
  std::vector<int> cnt((size_t)r->nfa);
  for (int f = 0; f < r->nfa; f++) cnt[f] = r->noofa_i[f + 1] - r->noofa_i[f];
  w.put(cnt.data(), 4 * cnt.size());
  w.put(r->noofa_v.data(), 4 * r->noofa_v.size());
  h = make_header("CVOFA", ID_CVOFA, kHeader + 8LL * r->nfa);
  h.idata[0] = r->nfa;
  h.idata[1] = 2;
  w.header(h);
  w.put(r->cvofa.data(), 4 * r->cvofa.size());
  for (const Zone& z : r->zones) {
    h = make_header(z.name.c_str(), ID_FA_ZONE, kHeader);
    h.idata[0] = z.kind;
    h.idata[1] = z.ifa_f;
    h.idata[2] = z.ifa_l;
    for (int k = 0; k < 3; k++) h.rdata[k] = z.periodic[k];
    w.header(h);
  }
  h = make_header("CV_PART", ID_CV_PART, kHeader + 4LL * r->ncv);
  h.idata[0] = r->ncv;
  h.idata[1] = r->nparts;
  w.header(h);
  w.put(r->cv_part.data(), 4 * r->cv_part.size());
  h = make_header("X_NO", ID_X_NO, kHeader + 24LL * r->nno);
  h.idata[0] = r->nno;
  h.idata[1] = 3;
  w.header(h);
  w.put(r->x_no.data(), 8 * r->x_no.size());
  w.header(make_header("DATA", ID_DATA, kHeader));
  for (int cls = 0; cls <= 4; cls++) {
    for (const Record& rec : r->records) {
      if (kind_class(rec.kind) != cls) continue;
      h = make_header(rec.name.c_str(), rec.kind, kHeader + 8LL * rec.count * rec.width);
      if (rec.kind == ID_I0) {
        h.idata[0] = rec.ivalue;
      } else if (rec.kind == ID_D0) {
        h.rdata[0] = rec.dvalue;
      } else {
        h.idata[0] = rec.count;
        if (rec.width >= 3) h.idata[1] = 3;
        if (rec.width == 9) h.idata[2] = 3;
      }
      w.header(h);
      if (rec.count) w.put(rec.data.data(), 8 * rec.data.size());
    }
  }
  w.header(make_header("EOF", ID_EOF, kHeader));
  FILE* f = std::fopen(path, "wb");
  if (!f) return set_err(JG_ERR_IO, std::string("cannot create restart file ") + path);
  const size_t put = std::fwrite(w.out.data(), 1, w.out.size(), f);
  const bool ok = put == w.out.size() && std::fclose(f) == 0;
  if (!ok) return set_err(JG_ERR_IO, std::string("cannot write restart file ") + path);
  return JG_OK;
}

int jg_restart_counts(const jg_restart_t* r, int* nno, int* nfa, int* ncv, int* noofa_count, int* nzones,
                      int* nrecords) {
  if (!r) return set_err(JG_ERR_ARG, "null restart");
  if (nno) *nno = r->nno;
  if (nfa) *nfa = r->nfa;
  if (ncv) *ncv = r->ncv;
  if (noofa_count) *noofa_count = r->noofa_count;
  if (nzones) *nzones = (int)r->zones.size();
  if (nrecords) *nrecords = (int)r->records.size();
  return JG_OK;
}

int jg_restart_get_mesh(const jg_restart_t* r, double* x_no, int* noofa_i, int* noofa_v, int* cvofa, int* cv_part) {
  if (!r) return set_err(JG_ERR_ARG, "null restart");
  if (x_no) std::memcpy(x_no, r->x_no.data(), 8 * r->x_no.size());
  if (noofa_i) std::memcpy(noofa_i, r->noofa_i.data(), 4 * r->noofa_i.size());
  if (noofa_v) std::memcpy(noofa_v, r->noofa_v.data(), 4 * r->noofa_v.size());
  if (cvofa) std::memcpy(cvofa, r->cvofa.data(), 4 * r->cvofa.size());
  if (cv_part) std::memcpy(cv_part, r->cv_part.data(), 4 * r->cv_part.size());
  return JG_OK;
}

int jg_restart_get_zone(const jg_restart_t* r, int izone, char* name, int* kind, int* ifa_f, int* ifa_l,
                        double* periodic) {
  if (!r) return set_err(JG_ERR_ARG, "null restart");
  if (izone < 0 || izone >= (int)r->zones.size()) return set_err(JG_ERR_ARG, "zone index out of range");
  const Zone& z = r->zones[izone];
  if (name) {
    std::memset(name, 0, kNameLen);
    std::strncpy(name, z.name.c_str(), kNameLen - 1);
  }
  if (kind) *kind = z.kind;
  if (ifa_f) *ifa_f = z.ifa_f;
  if (ifa_l) *ifa_l = z.ifa_l;
  if (periodic)
    for (int k = 0; k < 3; k++) periodic[k] = z.periodic[k];
  return JG_OK;
}

int jg_restart_set_mesh(jg_restart_t* r, int nno, int nfa, int ncv, const double* x_no, const int* noofa_i,
                        const int* noofa_v, const int* cvofa) {
  if (!r || nno < 0 || nfa < 0 || ncv < 0) return set_err(JG_ERR_ARG, "bad argument");
  if ((nno && !x_no) || (nfa && (!noofa_i || !cvofa))) return set_err(JG_ERR_ARG, "null mesh array");
  if (nfa && noofa_i[0] != 0) return set_err(JG_ERR_ARG, "noofa_i[0] must be 0");
  for (int f = 0; f < nfa; f++) {
    if (noofa_i[f + 1] < noofa_i[f]) return set_err(JG_ERR_ARG, "noofa_i must not decrease");
    if (cvofa[2 * f] < 0 || cvofa[2 * f] >= ncv || cvofa[2 * f + 1] >= ncv)
      return set_err(JG_ERR_ARG, "cvofa out of range at face %d", f);
  }
  const int nv = nfa ? noofa_i[nfa] : 0;
  if (nv && !noofa_v) return set_err(JG_ERR_ARG, "null noofa_v");
  for (int k = 0; k < nv; k++)
    if (noofa_v[k] < 0 || noofa_v[k] >= nno) return set_err(JG_ERR_ARG, "noofa_v out of range");
  for (const Record& rec : r->records) {
    const int n = (rec.kind == ID_FA_D1 || rec.kind == ID_FA_D3) ? nfa
                  : (rec.kind == ID_NO_D1 || rec.kind == ID_NO_D3) ? nno : ncv;
    if (rec.count && rec.count != n) return set_err(JG_ERR_ARG, "record '%s' does not fit the new mesh", rec.name.c_str());
  }
  r->nno = nno;
  r->nfa = nfa;
  r->ncv = ncv;
  r->noofa_count = nv;
  r->x_no.assign(x_no, x_no + 3 * (size_t)nno);
  r->noofa_i.assign((size_t)nfa + 1, 0);
  if (nfa) r->noofa_i.assign(noofa_i, noofa_i + nfa + 1);
  r->noofa_v.assign(noofa_v, noofa_v + nv);
  r->cvofa.assign(cvofa, cvofa + 2 * (size_t)nfa);
  r->cv_part.assign((size_t)ncv, 0);
  r->nparts = 1;
  r->zones.clear();
  r->has_mesh = true;
  return JG_OK;
}

int jg_restart_add_zone(jg_restart_t* r, const char* name, int kind, int ifa_f, int ifa_l, const double* periodic) {
  if (!r || !name) return set_err(JG_ERR_ARG, "null argument");
  if (std::strlen(name) >= (size_t)kNameLen) return set_err(JG_ERR_ARG, "zone name longer than 51 characters");
  if (kind < 1 || kind > 6) return set_err(JG_ERR_ARG, "zone kind %d (1..6: FA_ZONE_*)", kind);
  const int next = r->zones.empty() ? 0 : r->zones.back().ifa_l + 1;
  if (ifa_f != next || ifa_l < ifa_f - 1 || ifa_l >= r->nfa)
    return set_err(JG_ERR_ARG, "zone '%s' must start at face %d and end inside the mesh", name, next);
  Zone z;
  z.name = name;
  z.kind = kind;
  z.ifa_f = ifa_f;
  z.ifa_l = ifa_l;
  if (periodic)
    for (int k = 0; k < 3; k++) z.periodic[k] = periodic[k];
  r->zones.push_back(z);
  return JG_OK;
}

int jg_restart_find(const jg_restart_t* r, const char* name, int* irec) {
  if (!r || !name || !irec) return set_err(JG_ERR_ARG, "null argument");
  *irec = r->find(name);
  return JG_OK;
}

int jg_restart_get_record(const jg_restart_t* r, int irec, char* name, int* kind, int* count, int* width, double* data,
                          int* ivalue, double* dvalue) {
  if (!r) return set_err(JG_ERR_ARG, "null restart");
  if (irec < 0 || irec >= (int)r->records.size()) return set_err(JG_ERR_ARG, "record index out of range");
  const Record& rec = r->records[irec];
  if (name) {
    std::memset(name, 0, kNameLen);
    std::strncpy(name, rec.name.c_str(), kNameLen - 1);
  }
  if (kind) *kind = rec.kind;
  if (count) *count = rec.count;
  if (width) *width = rec.width;
  if (data && !rec.data.empty()) std::memcpy(data, rec.data.data(), 8 * rec.data.size());
  if (ivalue) *ivalue = rec.ivalue;
  if (dvalue) *dvalue = rec.dvalue;
  return JG_OK;
}

int jg_restart_put_record(jg_restart_t* r, const char* name, int kind, const double* data, int ivalue, double dvalue) {
  if (!r || !name) return set_err(JG_ERR_ARG, "null argument");
  if (std::strlen(name) >= (size_t)kNameLen || !*name) return set_err(JG_ERR_ARG, "record name must have 1..51 characters");
  const int w = kind_width(kind);
  if (w < 0) return set_err(JG_ERR_ARG, "record kind %d is not a data record", kind);
  Record rec;
  rec.name = name;
  rec.kind = kind;
  rec.width = w;
  rec.ivalue = kind == ID_I0 ? ivalue : 0;
  rec.dvalue = kind == ID_D0 ? dvalue : 0.0;
  if (w > 0) {
    if (!r->has_mesh) return set_err(JG_ERR_ARG, "set the mesh before array records");
    if (!data) return set_err(JG_ERR_ARG, "null data");
    rec.count = (kind == ID_FA_D1 || kind == ID_FA_D3) ? r->nfa : (kind == ID_NO_D1 || kind == ID_NO_D3) ? r->nno : r->ncv;
    rec.data.assign(data, data + (size_t)rec.count * w);
  }
  const int at = r->find(name);
  if (at >= 0) r->records[at] = std::move(rec);
  else r->records.push_back(std::move(rec));
  return JG_OK;
}

// The handle's conserved state, its transported scalars (nuSA; kine, omega:
// the names registerScalarTransport gives them, TurbModel_SA.h:31,
// TurbModel_KOMSST.h:38-47) and its step count (STEP, UgpWithCvCompFlow.h:307)
// into the restart, cells in the handle's caller order.
int jg_restart_save_state(jg_restart_t* r, jg_case_t* h) {
  if (!r || !h) return set_err(JG_ERR_ARG, "null argument");
  int ncv, nscal, turb, ncases;
  double cfl0;
  int rc = jg::case_restart_info(h, &ncv, &nscal, &turb, &ncases, &cfl0);
  if (rc) return rc;
  if (ncases != 1) return set_err(JG_ERR_ARG, "a batch handle holds several cases: save each case's state on its own");
  if (!r->has_mesh || r->ncv != ncv) return set_err(JG_ERR_ARG, "the restart's mesh has %d cells, the handle %d", r->ncv, ncv);
  std::vector<double> rho((size_t)ncv), rhou(3 * (size_t)ncv), rhoE((size_t)ncv);
  if ((rc = jg_get_state(h, rho.data(), rhou.data(), rhoE.data()))) return rc;
  double cfl;
  int step;
  if ((rc = jg_get_cfl_step(h, &cfl, &step))) return rc;
  jg_restart_put_record(r, "STEP", ID_I0, nullptr, step, 0.0);
  jg_restart_put_record(r, "RHO", ID_CV_D1, rho.data(), 0, 0.0);
  jg_restart_put_record(r, "RHOE", ID_CV_D1, rhoE.data(), 0, 0.0);
  if (nscal) {
    std::vector<double> phi((size_t)ncv * nscal), one((size_t)ncv);
    if ((rc = jg_get_scalars(h, phi.data()))) return rc;
    const char* names[2] = {turb == JG_TURB_SA ? "nuSA" : "kine", "omega"};
    for (int s = 0; s < nscal; s++) {
      for (int c = 0; c < ncv; c++) one[c] = phi[(size_t)c * nscal + s];
      jg_restart_put_record(r, names[s], ID_CV_D1, one.data(), 0, 0.0);
    }
  }
  return jg_restart_put_record(r, "RHOU", ID_CV_D3, rhou.data(), 0, 0.0);
}

// Sets the handle from the restart as readRestart + initialHook leave the
// reference (JoeWithModels.cpp:20-31, 201-213): RHO, RHOU, RHOE and the
// model's scalars, and the step count from STEP (0 if absent) with the CFL
// at its start value, so the CFL ramp of the following steps is the one
// runBackwardEuler takes after a restart (JoeWithModels.cpp:975-978).
int jg_restart_load_state(jg_case_t* h, const jg_restart_t* r) {
  if (!r || !h) return set_err(JG_ERR_ARG, "null argument");
  int ncv, nscal, turb, ncases;
  double cfl0;
  int rc = jg::case_restart_info(h, &ncv, &nscal, &turb, &ncases, &cfl0);
  if (rc) return rc;
  if (ncases != 1) return set_err(JG_ERR_ARG, "a batch handle holds several cases: load each case's state on its own");
  if (r->ncv != ncv) return set_err(JG_ERR_ARG, "the restart has %d cells, the handle %d", r->ncv, ncv);
  auto field = [&](const char* name, int kind) -> const Record* {
    const int i = r->find(name);
    if (i < 0 || r->records[i].kind != kind) return nullptr;
    return &r->records[i];
  };
  const Record* rho = field("RHO", ID_CV_D1);
  const Record* rhou = field("RHOU", ID_CV_D3);
  const Record* rhoE = field("RHOE", ID_CV_D1);
  if (!rho || !rhou || !rhoE) return set_err(JG_ERR_ARG, "the restart has no RHO, RHOU and RHOE cell records");
  if ((rc = jg_set_state(h, rho->data.data(), rhou->data.data(), rhoE->data.data()))) return rc;
  if (nscal) {
    const char* names[2] = {turb == JG_TURB_SA ? "nuSA" : "kine", "omega"};
    std::vector<double> phi((size_t)ncv * nscal);
    for (int s = 0; s < nscal; s++) {
      const Record* p = field(names[s], ID_CV_D1);
      if (!p) return set_err(JG_ERR_ARG, "the restart has no %s cell record", names[s]);
      for (int c = 0; c < ncv; c++) phi[(size_t)c * nscal + s] = p->data[c];
    }
    if ((rc = jg_set_scalars(h, phi.data()))) return rc;
  }
  const int i = r->find("STEP");
  const int step = (i >= 0 && r->records[i].kind == ID_I0) ? r->records[i].ivalue : 0;
  if (step < 0) return set_err(JG_ERR_ARG, "negative STEP in the restart");
  return jg_set_cfl_step(h, cfl0, step);
}

}  // extern "C"
