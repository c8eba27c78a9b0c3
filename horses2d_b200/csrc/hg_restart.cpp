// hg_restart.cpp -- restart files (*.HiORst) without a NetCDF library: the reference's Autosave
// (Solver/src/Approximation/DGTimeIntegrator.f90:413-454) writes, and DGSEM_loadRestartFile
// (Solver/src/Approximation/DGSEM_class.f90:263-291) reads, a NetCDF classic file with
//   dimensions  one = 1, NDOF, N, NCONS = 4, no_of_elements
//   variables   double t(one), double Q(NDOF), int iter(one)
// The classic format (CDF-1; CDF-2 is read too) is a big-endian header -- magic, record count,
// dimension list, global attributes, variable list with each variable's type, size and offset -- followed
// by the variables' data, each padded to 4 bytes.  The writer lays the file out in the reference's
// definition order with the data right after the header, as the reference's files are; the reader
// accepts any classic file holding those three variables.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

namespace {

thread_local std::string g_restart_err;   // per thread: asynchronous writes report on their own thread

enum : uint32_t { NC_DIMENSION = 10, NC_VARIABLE = 11, NC_ATTRIBUTE = 12, NC_INT = 4, NC_DOUBLE = 6 };

struct Out {
  std::vector<unsigned char> b;
  void u32(uint32_t v) { for (int s = 24; s >= 0; s -= 8) b.push_back(uint8_t(v >> s)); }
  void u64(uint64_t v) { for (int s = 56; s >= 0; s -= 8) b.push_back(uint8_t(v >> s)); }
  void name(const char* s) {
    const uint32_t n = uint32_t(std::strlen(s));
    u32(n);
    for (uint32_t i = 0; i < n; ++i) b.push_back(uint8_t(s[i]));
    while (b.size() % 4) b.push_back(0);
  }
  void f64(double v) { uint64_t u; std::memcpy(&u, &v, 8); u64(u); }
};

struct In {
  const unsigned char* p;
  size_t n, at = 0;
  void need(size_t k) const { if (at + k > n) throw std::runtime_error("truncated restart file"); }
  uint32_t u32() { need(4); uint32_t v = 0; for (int i = 0; i < 4; ++i) v = (v << 8) | p[at++]; return v; }
  uint64_t u64() { need(8); uint64_t v = 0; for (int i = 0; i < 8; ++i) v = (v << 8) | p[at++]; return v; }
  std::string name() {
    const uint32_t k = u32();
    need(k);
    std::string s(reinterpret_cast<const char*>(p + at), k);
    at += k;
    while (at % 4) ++at;
    return s;
  }
};

size_t type_size(uint32_t t) {
  switch (t) { case 1: case 2: return 1; case 3: return 2; case 4: case 5: return 4; case 6: return 8; default: break; }
  throw std::runtime_error("unknown NetCDF type in restart file");
}

void skip_attributes(In& in) {
  const uint32_t tag = in.u32(), n = in.u32();
  if (tag == 0 && n == 0) return;
  if (tag != NC_ATTRIBUTE) throw std::runtime_error("bad attribute list in restart file");
  for (uint32_t a = 0; a < n; ++a) {
    in.name();
    const uint32_t t = in.u32(), k = in.u32();
    size_t bytes = size_t(k) * type_size(t);
    bytes = (bytes + 3) / 4 * 4;
    in.need(bytes);
    in.at += bytes;
  }
}

struct Var {
  std::string name;
  uint32_t type = 0;
  uint64_t begin = 0, count = 1;
};

}  // namespace

extern "C" const char* hg_restart_last_error() { return g_restart_err.c_str(); }

extern "C" int hg_write_restart(const char* path, double t, int32_t iter, const double* Q, int64_t ndof, int32_t N,
                                int32_t n_elements) {
  try {
    if (!path || !Q || ndof < 4 || ndof % 4 || N < 1 || n_elements < 1) throw std::runtime_error("bad restart arguments");
    if (uint64_t(ndof) * 8 > 0xFFFFFFFFull) throw std::runtime_error("state too large for a classic (CDF-1) file");
    Out o;
    o.b.insert(o.b.end(), {'C', 'D', 'F', 1});
    o.u32(0);                                   // no record dimension
    o.u32(NC_DIMENSION); o.u32(5);
    const char* dn[5] = {"one", "NDOF", "N", "NCONS", "no_of_elements"};
    const uint32_t dl[5] = {1, uint32_t(ndof), uint32_t(N), 4, uint32_t(n_elements)};
    for (int d = 0; d < 5; ++d) { o.name(dn[d]); o.u32(dl[d]); }
    o.u32(0); o.u32(0);                         // no global attributes
    o.u32(NC_VARIABLE); o.u32(3);
    // header size is fixed by the names: compute the data offsets before writing them
    const size_t header = o.b.size() + 3 * (4 + 4 + 4 + 4 + 4 + 4 + 4 + 4) + 4 /*"t"*/ + 4 /*"Q"*/ + 4 /*"iter"*/;
    const uint32_t vsize_q = uint32_t(ndof) * 8;
    const uint32_t begin_t = uint32_t(header), begin_q = begin_t + 8, begin_i = begin_q + vsize_q;
    auto var = [&](const char* nm, uint32_t dim, uint32_t type, uint32_t vsize, uint32_t begin) {
      o.name(nm); o.u32(1); o.u32(dim); o.u32(0); o.u32(0); o.u32(type); o.u32(vsize); o.u32(begin);
    };
    var("t", 0, NC_DOUBLE, 8, begin_t);
    var("Q", 1, NC_DOUBLE, vsize_q, begin_q);
    var("iter", 0, NC_INT, 4, begin_i);
    if (o.b.size() != header) throw std::runtime_error("restart header size mismatch");
    o.f64(t);
    for (int64_t i = 0; i < ndof; ++i) o.f64(Q[i]);
    o.u32(uint32_t(iter));
    FILE* f = std::fopen(path, "wb");
    if (!f) throw std::runtime_error(std::string("cannot open ") + path);
    const size_t w = std::fwrite(o.b.data(), 1, o.b.size(), f);
    const int c = std::fclose(f);
    if (w != o.b.size() || c != 0) throw std::runtime_error(std::string("cannot write ") + path);
    g_restart_err.clear();
    return 0;
  } catch (const std::exception& ex) {
    g_restart_err = ex.what();
    return 1;
  }
}

extern "C" int hg_read_restart(const char* path, double* t, int32_t* iter, double* Q, int64_t capacity,
                               int64_t* ndof) {
  try {
    if (!path) throw std::runtime_error("bad restart arguments");
    FILE* f = std::fopen(path, "rb");
    if (!f) throw std::runtime_error(std::string("cannot open ") + path);
    std::vector<unsigned char> buf;
    unsigned char chunk[1 << 16];
    size_t r;
    while ((r = std::fread(chunk, 1, sizeof(chunk), f)) > 0) buf.insert(buf.end(), chunk, chunk + r);
    std::fclose(f);
    In in{buf.data(), buf.size()};
    in.need(4);
    if (std::memcmp(buf.data(), "CDF", 3) != 0 || (buf[3] != 1 && buf[3] != 2))
      throw std::runtime_error("not a NetCDF classic file");
    const bool offset64 = buf[3] == 2;
    in.at = 4;
    in.u32();                                   // record count (unused: no record variables here)
    std::vector<uint64_t> dims;
    {
      const uint32_t tag = in.u32(), n = in.u32();
      if (!(tag == 0 && n == 0)) {
        if (tag != NC_DIMENSION) throw std::runtime_error("bad dimension list in restart file");
        for (uint32_t d = 0; d < n; ++d) { in.name(); dims.push_back(in.u32()); }
      }
    }
    skip_attributes(in);
    std::vector<Var> vars;
    {
      const uint32_t tag = in.u32(), n = in.u32();
      if (!(tag == 0 && n == 0)) {
        if (tag != NC_VARIABLE) throw std::runtime_error("bad variable list in restart file");
        for (uint32_t v = 0; v < n; ++v) {
          Var x;
          x.name = in.name();
          const uint32_t nd = in.u32();
          for (uint32_t d = 0; d < nd; ++d) {
            const uint32_t id = in.u32();
            if (id >= dims.size()) throw std::runtime_error("bad dimension id in restart file");
            x.count *= dims[id];
          }
          skip_attributes(in);
          x.type = in.u32();
          in.u32();                             // vsize
          x.begin = offset64 ? in.u64() : in.u32();
          vars.push_back(x);
        }
      }
    }
    auto find = [&](const char* nm) -> const Var& {
      for (const Var& v : vars) if (v.name == nm) return v;
      throw std::runtime_error(std::string("restart file has no variable ") + nm);
    };
    auto read_f64 = [&](const Var& v, uint64_t i) {
      In at{buf.data(), buf.size(), size_t(v.begin + 8 * i)};
      const uint64_t u = at.u64();
      double d;
      std::memcpy(&d, &u, 8);
      return d;
    };
    const Var& vt = find("t");
    const Var& vq = find("Q");
    const Var& vi = find("iter");
    if (vt.type != NC_DOUBLE || vq.type != NC_DOUBLE || vi.type != NC_INT)
      throw std::runtime_error("restart variables have unexpected types");
    if (ndof) *ndof = int64_t(vq.count);
    if (t) *t = read_f64(vt, 0);
    if (iter) { In at{buf.data(), buf.size(), size_t(vi.begin)}; *iter = int32_t(at.u32()); }
    if (Q) {
      if (int64_t(vq.count) > capacity) throw std::runtime_error("restart state larger than the buffer");
      for (uint64_t i = 0; i < vq.count; ++i) Q[i] = read_f64(vq, i);
    }
    g_restart_err.clear();
    return 0;
  } catch (const std::exception& ex) {
    g_restart_err = ex.what();
    return 1;
  }
}

// ---- the resident state of a context to and from a restart file -------------------------------------
// The state layout Q[e][eta][xi][var] is the reference's Storage%Q, so the file's Q is copied as is.
extern "C" {
int hg_get_state(struct hg_ctx* ctx, double* Q, int64_t ndof);
int hg_set_state(struct hg_ctx* ctx, const double* Q, int64_t ndof);
int64_t hg_ndof(const struct hg_ctx* ctx);
int hg_info(const struct hg_ctx* ctx, int32_t out[4]);
const char* hg_last_error(const struct hg_ctx* ctx);
}

extern "C" int hg_save_restart(struct hg_ctx* ctx, const char* path, double t, int32_t iter) {
  int32_t info[4];
  const int64_t ndof = ctx ? hg_ndof(ctx) : 0;
  if (!ctx || ndof <= 0 || hg_info(ctx, info) != 0) { g_restart_err = "bad context"; return 1; }
  std::vector<double> Q(static_cast<size_t>(ndof));
  if (hg_get_state(ctx, Q.data(), ndof) != 0) { g_restart_err = hg_last_error(ctx); return 1; }
  return hg_write_restart(path, t, iter, Q.data(), ndof, info[0], info[1]);
}

extern "C" int hg_load_restart(struct hg_ctx* ctx, const char* path, double* t, int32_t* iter) {
  const int64_t ndof = ctx ? hg_ndof(ctx) : 0;
  if (!ctx || ndof <= 0) { g_restart_err = "bad context"; return 1; }
  int64_t n = 0;
  if (hg_read_restart(path, nullptr, nullptr, nullptr, 0, &n) != 0) return 1;
  if (n != ndof) {
    g_restart_err = "restart file holds " + std::to_string(n) + " values, the context " + std::to_string(ndof);
    return 1;
  }
  std::vector<double> Q(static_cast<size_t>(ndof));
  if (hg_read_restart(path, t, iter, Q.data(), ndof, nullptr) != 0) return 1;
  if (hg_set_state(ctx, Q.data(), ndof) != 0) { g_restart_err = hg_last_error(ctx); return 1; }
  return 0;
}
