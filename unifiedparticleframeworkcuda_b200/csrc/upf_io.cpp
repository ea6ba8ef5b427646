// upf_io.cpp — particle state files.
//
// * The reference's text formats, byte for byte: the writers of
//   UnifiedIO (src/cpu/UnifiedIO.cpp:14-152) and Scene::saveParticles
//   (src/sceneConfigure/Scene.cpp:247-279), and the readers
//   UnifiedIO::ReadInFluidParticleNum / ReadInFluidParticlesPCISPH
//   (UnifiedIO.cpp:154-220) and Scene::readInParticles (Scene.cpp:218-243).
//   The reference formats through std::ofstream (precision, setw, left) and
//   parses with operator>>; here every record is formatted with the same
//   printf conversion the stream uses (libstdc++ formats a double with
//   "%.*g" and pads to the field width), in contiguous chunks on worker
//   threads that are written out in order, and parsed by a scanner that
//   accepts exactly what the stream's extraction accepts.
// * A binary snapshot file: upf_state_save's bytes behind a header that
//   records the format, the system's parameters and counts, and a checksum,
//   so a run can stop and resume in another process bit for bit.
//
// Host code only: the particle data comes from the caller's arrays or from
// the device through the public readback calls.
#include <locale.h>

#include <algorithm>
#include <cerrno>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstddef>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/upf.h"
#include "upf_internal.h"

namespace upf {
namespace {

// ---------------------------------------------------------------- formatting
// Every conversion runs in the "C" locale (decimal point '.'), as the
// reference's streams do, whatever locale the host process has set.
struct CLocaleScope {
  locale_t c = (locale_t)0, prev = (locale_t)0;
  CLocaleScope() {
    c = newlocale(LC_ALL_MASK, "C", (locale_t)0);
    if (c) prev = uselocale(c);
  }
  ~CLocaleScope() {
    if (c) {
      uselocale(prev);
      freelocale(c);
    }
  }
};

unsigned io_workers(size_t records) {
  unsigned hw = std::thread::hardware_concurrency();
  if (hw == 0) hw = 1;
  const size_t by_size = records / 16384 + 1;  // at least 16k records per worker
  return (unsigned)std::min<size_t>({(size_t)hw, by_size, (size_t)64});
}

// Formats records [0, n) into one string per worker (contiguous ranges, in
// order). rec(i, buf) writes record i into buf (at most kRecordMax bytes)
// and returns its length, or 0 to skip the record.
constexpr int kRecordMax = 512;

template <class Rec>
std::vector<std::string> format_chunks(size_t n, Rec&& rec) {
  const unsigned w = io_workers(n);
  std::vector<std::string> out(w);
  auto work = [&](unsigned t) {
    CLocaleScope loc;
    const size_t b = n * t / w, e = n * (t + 1) / w;
    std::string& s = out[t];
    s.reserve((e - b) * 96);
    char buf[kRecordMax];
    for (size_t i = b; i < e; ++i) {
      const int len = rec(i, buf);
      if (len > 0) s.append(buf, (size_t)len);
    }
  };
  if (w == 1) {
    work(0);
  } else {
    std::vector<std::thread> th;
    th.reserve(w);
    for (unsigned t = 0; t < w; ++t) th.emplace_back(work, t);
    for (auto& x : th) x.join();
  }
  return out;
}

upf_status write_file(const char* path, const std::string& head, const std::vector<std::string>& body,
                      const std::string& tail, const char* who) {
  FILE* f = std::fopen(path, "wb");
  if (!f) {
    set_error("%s: cannot open %s for writing: %s", who, path, std::strerror(errno));
    return UPF_ERR_IO;
  }
  bool ok = std::fwrite(head.data(), 1, head.size(), f) == head.size();
  for (const auto& s : body) ok = ok && std::fwrite(s.data(), 1, s.size(), f) == s.size();
  ok = ok && std::fwrite(tail.data(), 1, tail.size(), f) == tail.size();
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) {
    set_error("%s: writing %s failed: %s", who, path, std::strerror(errno));
    return UPF_ERR_IO;
  }
  return UPF_OK;
}

std::string fmt_line(const char* fmt, long long v) {
  CLocaleScope loc;
  char buf[64];
  const int len = std::snprintf(buf, sizeof buf, fmt, v);
  return std::string(buf, (size_t)len);
}

// One record of SaveLiquidParticleInfoFull / SaveRigidParticleInfoFull
// (UnifiedIO.cpp:84-96, 131-143): precision(8), left-aligned, widths 15 / 3
// / 15 / 2; only the position and type carry data, the other fields are the
// zeros the reference writes.
int info_record(char* buf, const float* p4, int type) {
  return std::snprintf(buf, kRecordMax, "%-15.8g %-15.8g %-15.8g %-3d %-15.8g %.8g %.8g %-2.8g %-2.8g %-2.8g %-2.8g \n",
                       (double)p4[0], (double)p4[1], (double)p4[2], type, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0);
}

upf_status save_info_full(const char* path, const float* pos4, const int32_t* type, int32_t num_rounded,
                          int32_t header_count, bool rigid, const char* who) {
  if (!path || num_rounded < 0 || (num_rounded > 0 && (!pos4 || !type))) {
    set_error("%s: bad arguments", who);
    return UPF_ERR_INVALID_ARG;
  }
  auto body = format_chunks((size_t)num_rounded, [&](size_t i, char* buf) {
    const int t = type[i];
    const bool take = rigid ? (t == UPF_RIGID || t == UPF_FROZEN) : (t == UPF_LIQUID);
    return take ? info_record(buf, pos4 + 4 * i, t) : 0;
  });
  return write_file(path, fmt_line("%lld\n", header_count), body, std::string(), who);
}

}  // namespace
}  // namespace upf

using namespace upf;

// UnifiedIO::SaveLiquidParticleInfoFull (UnifiedIO.cpp:60-105)
upf_status upf_io_save_liquid_info_full(const char* path, const float* pos4, const int32_t* type,
                                        int32_t num_rounded_particles, int32_t num_liquid_particles) {
  return save_info_full(path, pos4, type, num_rounded_particles, num_liquid_particles, false,
                        "upf_io_save_liquid_info_full");
}

// UnifiedIO::SaveRigidParticleInfoFull (UnifiedIO.cpp:107-152)
upf_status upf_io_save_rigid_info_full(const char* path, const float* pos4, const int32_t* type,
                                       int32_t num_rounded_particles, int32_t header_count) {
  return save_info_full(path, pos4, type, num_rounded_particles, header_count, true, "upf_io_save_rigid_info_full");
}

// UnifiedIO::SaveParticlePositions (UnifiedIO.cpp:14-58): the count, then per
// particle its position at precision(20) and eight zeros.
upf_status upf_io_save_particle_positions(const char* path, const float* pos4, uint32_t n) {
  if (!path || (n > 0 && !pos4)) {
    set_error("upf_io_save_particle_positions: bad arguments");
    return UPF_ERR_INVALID_ARG;
  }
  auto body = format_chunks(n, [&](size_t i, char* buf) {
    const float* p = pos4 + 4 * i;
    return std::snprintf(buf, kRecordMax, "%.20g %.20g %.20g %.20g %.20g %.20g %.20g %.20g %.20g %.20g %.20g \n",
                         (double)p[0], (double)p[1], (double)p[2], 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0);
  });
  return write_file(path, fmt_line("%lld\n", (long long)n), body, std::string(), "upf_io_save_particle_positions");
}

// Scene::saveParticles (Scene.cpp:247-279): per particle position, rest
// density, mass and type (written as a float) at the default precision, then
// one empty line. rest_density / mass may be NULL (one value for all).
upf_status upf_io_save_scene_particles(const char* path, const float* pos4, const float* rest_density,
                                       const float* mass, const int32_t* type, uint32_t n, float rest_density_all,
                                       float mass_all) {
  if (!path || (n > 0 && (!pos4 || !type))) {
    set_error("upf_io_save_scene_particles: bad arguments");
    return UPF_ERR_INVALID_ARG;
  }
  auto body = format_chunks(n, [&](size_t i, char* buf) {
    const float* p = pos4 + 4 * i;
    const float rd = rest_density ? rest_density[i] : rest_density_all;
    const float m = mass ? mass[i] : mass_all;
    return std::snprintf(buf, kRecordMax, "%g %g %g %g %g %g \n", (double)p[0], (double)p[1], (double)p[2],
                         (double)rd, (double)m, (double)(float)type[i]);
  });
  return write_file(path, std::string(), body, std::string("\n"), "upf_io_save_scene_particles");
}

// The file UnifiedIO::ReadInFluidParticlesPCISPH reads (UnifiedIO.cpp:179-220;
// the reference's own writer for it, SaveLiquidParticleInfoForLoading, is
// referenced at UnifiedPhysics.cpp:6181 but not in the sources): the count,
// then per particle position, type, velocity, correction pressure and
// predicted density, at 9 significant digits (every float reads back exactly).
upf_status upf_io_save_fluid_particles_pcisph(const char* path, const float* pos4, const float* vel4,
                                              const int32_t* type, const float* corr_pressure,
                                              const float* predicted_density, uint32_t n) {
  if (!path || (n > 0 && (!pos4 || !vel4 || !type))) {
    set_error("upf_io_save_fluid_particles_pcisph: bad arguments");
    return UPF_ERR_INVALID_ARG;
  }
  auto body = format_chunks(n, [&](size_t i, char* buf) {
    const float* p = pos4 + 4 * i;
    const float* v = vel4 + 4 * i;
    const double pc = corr_pressure ? (double)corr_pressure[i] : 0.0;
    const double rs = predicted_density ? (double)predicted_density[i] : 0.0;
    return std::snprintf(buf, kRecordMax, "%.9g %.9g %.9g %d %.9g %.9g %.9g %.9g %.9g\n", (double)p[0], (double)p[1],
                         (double)p[2], type[i], (double)v[0], (double)v[1], (double)v[2], pc, rs);
  });
  return write_file(path, fmt_line("%lld\n", (long long)n), body, std::string(), "upf_io_save_fluid_particles_pcisph");
}

// ---------------------------------------------------------------- parsing
namespace upf {
namespace {

// Reads a whole file into memory.
upf_status slurp(const char* path, std::string& out, const char* who) {
  if (!path) {
    set_error("%s: null path", who);
    return UPF_ERR_INVALID_ARG;
  }
  FILE* f = std::fopen(path, "rb");
  if (!f) {
    set_error("%s: cannot open %s: %s", who, path, std::strerror(errno));
    return UPF_ERR_IO;
  }
  out.clear();
  if (std::fseek(f, 0, SEEK_END) == 0) {
    const long size = std::ftell(f);
    if (size > 0) out.reserve((size_t)size);
    std::rewind(f);
  }
  char buf[1 << 16];
  size_t got;
  while ((got = std::fread(buf, 1, sizeof buf, f)) > 0) out.append(buf, got);
  const bool err = std::ferror(f) != 0;
  std::fclose(f);
  if (err) {
    set_error("%s: reading %s failed", who, path);
    return UPF_ERR_IO;
  }
  return UPF_OK;
}

// Formatted extraction as std::istream's operator>> does it in the "C"
// locale (libstdc++ num_get): skip white space; an int is an optional sign
// and decimal digits; a float is an optional sign, digits with at most one
// decimal point, and an exponent (e/E, optional sign, digits) after at least
// one mantissa digit, converted with strtof. A field that matches nothing,
// does not convert as a whole, or overflows fails (the stream's failbit),
// and so does the end of the input.
bool is_space(char c) { return c == ' ' || c == '\t' || c == '\n' || c == '\v' || c == '\f' || c == '\r'; }
bool is_digit(char c) { return c >= '0' && c <= '9'; }

// One int field starting at p (white space already skipped); advances p past
// what the field took.
bool scan_int(const char*& p, const char* end, int32_t& v) {
  const char* q = p;
  bool neg = false;
  if (q < end && (*q == '+' || *q == '-')) neg = *q++ == '-';
  long long acc = 0;
  bool any = false, big = false;
  while (q < end && is_digit(*q)) {
    acc = acc * 10 + (*q++ - '0');
    any = true;
    if (acc > (long long)INT_MAX + 1) big = true, acc = (long long)INT_MAX + 1;
  }
  p = q;
  if (!any) return false;
  if (neg) acc = -acc;
  if (big || acc > INT_MAX || acc < INT_MIN) return false;
  v = (int32_t)acc;
  return true;
}

// One float field starting at p (white space already skipped).
bool scan_float(const char*& p, const char* end, float& v) {
  const char* q = p;
  if (q < end && (*q == '+' || *q == '-')) ++q;
  bool mant = false, dec = false, sci = false;
  while (q < end) {
    const char c = *q;
    if (is_digit(c)) {
      if (!sci) mant = true;
      ++q;
    } else if (c == '.' && !dec && !sci) {
      dec = true;
      ++q;
    } else if ((c == 'e' || c == 'E') && mant && !sci) {
      sci = true;
      ++q;
      if (q < end && (*q == '+' || *q == '-')) ++q;
    } else {
      break;
    }
  }
  const size_t len = (size_t)(q - p);
  const char* tok = p;
  p = q;
  if (len == 0) return false;
  char small[128];
  std::string big;
  const char* z;
  if (len < sizeof small) {
    std::memcpy(small, tok, len);
    small[len] = '\0';
    z = small;
  } else {
    big.assign(tok, len);
    z = big.c_str();
  }
  char* stop = nullptr;
  const float x = std::strtof(z, &stop);
  if (stop != z + len || std::isinf(x)) return false;
  v = x;
  return true;
}

struct Scanner {
  const char* p;
  const char* end;
  const char* begin;

  explicit Scanner(const std::string& s) : p(s.data()), end(s.data() + s.size()), begin(s.data()) {}

  // true when only white space is left (a clean end of the records)
  bool at_end() {
    while (p < end && is_space(*p)) ++p;
    return p == end;
  }
  bool get_int(int32_t& v) { return !at_end() && scan_int(p, end, v); }
  bool get_float(float& v) { return !at_end() && scan_float(p, end, v); }
  size_t offset() const { return (size_t)(p - begin); }
};

// Records of a fixed field layout (`kinds`: 'f' / 'i' per field, repeating)
// in [b, e), parsed on several threads. The text is cut into chunks at white
// space; each worker counts the white-space separated tokens of its chunk,
// then parses each token as the field its global index falls on. floats go
// to fl[record * nf + k], ints to in[record * ni + k] (k counting fields of
// that kind). Returns false, with nothing promised about the outputs, when a
// token is not exactly one field of its kind (operator>> would split or
// reject it: the sequential scanner then reads the file), or when the token
// count is not `records` full records (records == 0: any whole number of
// records, returned in *records_out).
bool parse_records_parallel(const char* b, const char* e, const char* kinds, size_t records, std::vector<float>& fl,
                            std::vector<int32_t>& in, size_t* records_out) {
  const size_t period = std::strlen(kinds);
  size_t nf = 0, ni = 0;
  std::vector<int> slot(period);
  for (size_t k = 0; k < period; ++k) slot[k] = kinds[k] == 'f' ? (int)nf++ : (int)ni++;
  const size_t bytes = (size_t)(e - b);
  const unsigned w = (unsigned)std::max<size_t>(1, std::min<size_t>(io_workers(bytes / 48), 64));
  std::vector<const char*> cut(w + 1);
  cut[0] = b;
  cut[w] = e;
  for (unsigned t = 1; t < w; ++t) {
    const char* c = b + bytes * t / w;
    if (c < cut[t - 1]) c = cut[t - 1];
    while (c < e && !is_space(*c)) ++c;  // never split a token
    cut[t] = c;
  }
  std::vector<size_t> count(w + 1, 0);
  auto run = [&](auto&& fn) {
    if (w == 1) {
      fn(0u);
      return;
    }
    std::vector<std::thread> th;
    for (unsigned t = 0; t < w; ++t) th.emplace_back(fn, t);
    for (auto& x : th) x.join();
  };
  run([&](unsigned t) {
    size_t n = 0;
    for (const char* c = cut[t]; c < cut[t + 1];) {
      while (c < cut[t + 1] && is_space(*c)) ++c;
      if (c == cut[t + 1]) break;
      ++n;
      while (c < cut[t + 1] && !is_space(*c)) ++c;
    }
    count[t + 1] = n;
  });
  for (unsigned t = 0; t < w; ++t) count[t + 1] += count[t];
  const size_t tokens = count[w];
  if (records == 0) {
    if (tokens % period) return false;
    records = tokens / period;
  } else if (tokens < records * period) {
    return false;
  }
  fl.assign(records * nf, 0.0f);
  in.assign(records * ni, 0);
  const size_t need = records * period;
  std::vector<char> bad(w, 0);
  run([&](unsigned t) {
    CLocaleScope loc;
    size_t g = count[t];
    for (const char* c = cut[t]; c < cut[t + 1] && g < need;) {
      while (c < cut[t + 1] && is_space(*c)) ++c;
      if (c == cut[t + 1]) break;
      const char* tok_end = c;
      while (tok_end < cut[t + 1] && !is_space(*tok_end)) ++tok_end;
      const size_t rec = g / period, k = g % period;
      const char* q = c;
      bool ok;
      if (kinds[k] == 'f') {
        ok = scan_float(q, tok_end, fl[rec * nf + (size_t)slot[k]]);
      } else {
        ok = scan_int(q, tok_end, in[rec * ni + (size_t)slot[k]]);
      }
      if (!ok || q != tok_end) {
        bad[t] = 1;
        return;
      }
      c = tok_end;
      ++g;
    }
  });
  for (char x : bad)
    if (x) return false;
  if (records_out) *records_out = records;
  return true;
}

}  // namespace
}  // namespace upf

// UnifiedIO::ReadInFluidParticleNum (UnifiedIO.cpp:154-177): the leading count.
upf_status upf_io_read_fluid_particle_num(const char* path, int32_t* count) {
  if (!count) {
    set_error("upf_io_read_fluid_particle_num: null count");
    return UPF_ERR_INVALID_ARG;
  }
  // only the head of the file: white space, then the count's characters
  if (!path) {
    set_error("upf_io_read_fluid_particle_num: null path");
    return UPF_ERR_INVALID_ARG;
  }
  FILE* f = std::fopen(path, "rb");
  if (!f) {
    set_error("upf_io_read_fluid_particle_num: cannot open %s: %s", path, std::strerror(errno));
    return UPF_ERR_IO;
  }
  std::string buf;
  for (int c; (c = std::fgetc(f)) != EOF;) {
    const bool sp = is_space((char)c);
    if (!sp) buf.push_back((char)c);
    if ((sp && !buf.empty()) || buf.size() > 32) break;
  }
  std::fclose(f);
  CLocaleScope loc;
  Scanner sc(buf);
  int32_t n = 0;
  if (!sc.get_int(n)) {
    set_error("upf_io_read_fluid_particle_num: %s does not start with a particle count", path);
    return UPF_ERR_IO;
  }
  *count = n;
  return UPF_OK;
}

// UnifiedIO::ReadInFluidParticlesPCISPH (UnifiedIO.cpp:179-220): the count,
// then that many records of position (3), type, velocity (3), correction
// pressure and predicted density, into arrays of `capacity` particles
// (pos3 / vel3: 3 floats per particle, as the reference's). The reference
// keeps a record whose fields stopped parsing half way and stops after it;
// here *n_read counts the complete records and an incomplete one is an error.
upf_status upf_io_read_fluid_particles_pcisph(const char* path, float* pos3, float* vel3, int32_t* type,
                                              float* corr_pressure, float* predicted_density, int32_t capacity,
                                              int32_t* n_read) {
  const char* who = "upf_io_read_fluid_particles_pcisph";
  if (!n_read || capacity < 0 || (capacity > 0 && (!pos3 || !vel3 || !type || !corr_pressure || !predicted_density))) {
    set_error("%s: bad arguments", who);
    return UPF_ERR_INVALID_ARG;
  }
  *n_read = 0;
  std::string buf;
  upf_status st = slurp(path, buf, who);
  if (st != UPF_OK) return st;
  CLocaleScope loc;
  Scanner sc(buf);
  int32_t cnt = 0;
  if (!sc.get_int(cnt) || cnt < 0) {
    set_error("%s: %s does not start with a particle count", who, path);
    return UPF_ERR_IO;
  }
  if (cnt > capacity) {
    set_error("%s: %s holds %d particles, capacity is %d", who, path, cnt, capacity);
    return UPF_ERR_INVALID_ARG;
  }
  std::vector<float> fl;
  std::vector<int32_t> in;
  if (cnt > 0 && parse_records_parallel(sc.p, sc.end, "fffifffff", (size_t)cnt, fl, in, nullptr)) {
    for (int32_t i = 0; i < cnt; ++i) {
      const float* f = &fl[(size_t)i * 8];
      for (int a = 0; a < 3; ++a) {
        pos3[3 * i + a] = f[a];
        vel3[3 * i + a] = f[3 + a];
      }
      type[i] = in[(size_t)i];
      corr_pressure[i] = f[6];
      predicted_density[i] = f[7];
    }
    *n_read = cnt;
    return UPF_OK;
  }
  for (int32_t i = 0; i < cnt; ++i) {
    float f[8];
    int32_t t = 0;
    const bool ok = sc.get_float(f[0]) && sc.get_float(f[1]) && sc.get_float(f[2]) && sc.get_int(t) &&
                    sc.get_float(f[3]) && sc.get_float(f[4]) && sc.get_float(f[5]) && sc.get_float(f[6]) &&
                    sc.get_float(f[7]);
    if (!ok) {
      set_error("%s: %s: record %d of %d is incomplete or malformed (byte %zu)", who, path, i, cnt, sc.offset());
      return UPF_ERR_IO;
    }
    pos3[3 * i] = f[0];
    pos3[3 * i + 1] = f[1];
    pos3[3 * i + 2] = f[2];
    type[i] = t;
    vel3[3 * i] = f[3];
    vel3[3 * i + 1] = f[4];
    vel3[3 * i + 2] = f[5];
    corr_pressure[i] = f[6];
    predicted_density[i] = f[7];
    *n_read = i + 1;
  }
  return UPF_OK;
}

// Scene::readInParticles (Scene.cpp:218-243): records of position, density,
// mass and type up to the end of the file; granular records (type 3) are
// skipped, as there. The reference's loop tests the stream before reading,
// so at the end of the file it adds the last record a second time; here a
// record is kept only when all its fields were read, and a file that ends
// in the middle of a record is an error. With NULL arrays only the count of
// kept records is returned (in *n_out); otherwise at most `capacity` are
// stored (pos4: x, y, z, 0).
upf_status upf_io_read_scene_particles(const char* path, float* pos4, float* density, float* mass, int32_t* type,
                                       uint32_t capacity, uint32_t* n_out) {
  const char* who = "upf_io_read_scene_particles";
  const bool fill = pos4 || density || mass || type;
  if (!n_out || (fill && (!pos4 || !density || !mass || !type))) {
    set_error("%s: bad arguments (all four arrays, or none to count)", who);
    return UPF_ERR_INVALID_ARG;
  }
  *n_out = 0;
  std::string buf;
  upf_status st = slurp(path, buf, who);
  if (st != UPF_OK) return st;
  CLocaleScope loc;
  Scanner sc(buf);
  uint32_t kept = 0;
  std::vector<float> fl;
  std::vector<int32_t> in;
  size_t nrec = 0;
  if (parse_records_parallel(sc.p, sc.end, "fffffi", 0, fl, in, &nrec)) {
    for (size_t r = 0; r < nrec; ++r) {
      if (in[r] == UPF_GRANULAR) continue;
      if (fill) {
        if (kept >= capacity) {
          set_error("%s: %s holds more than capacity %u particles", who, path, capacity);
          return UPF_ERR_INVALID_ARG;
        }
        const float* f = &fl[r * 5];
        pos4[4 * kept] = f[0];
        pos4[4 * kept + 1] = f[1];
        pos4[4 * kept + 2] = f[2];
        pos4[4 * kept + 3] = 0.0f;
        density[kept] = f[3];
        mass[kept] = f[4];
        type[kept] = in[r];
      }
      ++kept;
    }
    *n_out = kept;
    return UPF_OK;
  }
  while (!sc.at_end()) {
    float x, y, z, d, m;
    int32_t t = 0;
    const bool ok = sc.get_float(x) && sc.get_float(y) && sc.get_float(z) && sc.get_float(d) && sc.get_float(m) &&
                    sc.get_int(t);
    if (!ok) {
      set_error("%s: %s: record after %u kept particles is incomplete or malformed (byte %zu)", who, path, kept,
                sc.offset());
      return UPF_ERR_IO;
    }
    if (t == UPF_GRANULAR) continue;
    if (fill) {
      if (kept >= capacity) {
        set_error("%s: %s holds more than capacity %u particles", who, path, capacity);
        return UPF_ERR_INVALID_ARG;
      }
      pos4[4 * kept] = x;
      pos4[4 * kept + 1] = y;
      pos4[4 * kept + 2] = z;
      pos4[4 * kept + 3] = 0.0f;
      density[kept] = d;
      mass[kept] = m;
      type[kept] = t;
    }
    ++kept;
  }
  *n_out = kept;
  return UPF_OK;
}

// ---------------------------------------------------------------- snapshot file
// Layout: StateFileHeader, the saving system's upf_params, then the
// upf_state_save bytes. The checksum is FNV-1a (64 bit) over the parameters
// and the state bytes.
namespace upf {
namespace {

constexpr char kStateMagic[8] = {'U', 'P', 'F', 'S', 'T', 'A', 'T', 'E'};
constexpr uint32_t kStateVersion = 1;

struct StateFileHeader {
  char magic[8];
  uint32_t version;
  uint32_t abi_version;
  uint32_t header_bytes;   // sizeof(StateFileHeader)
  uint32_t params_bytes;   // sizeof(upf_params)
  uint64_t state_bytes;
  uint64_t checksum;
  uint32_t n_dynamic;
  uint32_t num_bodies;
  int32_t method;
  uint32_t reserved[3];
};
static_assert(sizeof(StateFileHeader) == 64, "snapshot header layout");

uint64_t fnv1a(const void* data, size_t n, uint64_t h = 0xcbf29ce484222325ull) {
  const unsigned char* p = static_cast<const unsigned char*>(data);
  for (size_t i = 0; i < n; ++i) h = (h ^ p[i]) * 0x100000001b3ull;
  return h;
}

upf_status system_counts(upf_system* s, uint32_t* n_dyn, uint32_t* bodies) {
  upf_status st = upf_get_particles(s, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, n_dyn);
  if (st != UPF_OK) return st;
  return upf_get_rigid_bodies(s, nullptr, nullptr, nullptr, nullptr, bodies);
}

upf_status read_header(FILE* f, const char* path, StateFileHeader& h, upf_params& prm, const char* who) {
  if (std::fread(&h, sizeof h, 1, f) != 1 || std::memcmp(h.magic, kStateMagic, 8) != 0) {
    set_error("%s: %s is not a particle state file", who, path);
    return UPF_ERR_IO;
  }
  if (h.version != kStateVersion || h.header_bytes != sizeof(StateFileHeader) ||
      h.params_bytes != sizeof(upf_params)) {
    set_error("%s: %s has format version %u (header %u B, parameters %u B); this library reads version %u (%zu B, %zu B)",
              who, path, h.version, h.header_bytes, h.params_bytes, kStateVersion, sizeof(StateFileHeader),
              sizeof(upf_params));
    return UPF_ERR_IO;
  }
  if (std::fread(&prm, sizeof prm, 1, f) != 1) {
    set_error("%s: %s is truncated", who, path);
    return UPF_ERR_IO;
  }
  return UPF_OK;
}

}  // namespace
}  // namespace upf

upf_status upf_state_write_file(upf_system* s, const char* path) {
  const char* who = "upf_state_write_file";
  if (!s || !path) {
    set_error("%s: null argument", who);
    return UPF_ERR_INVALID_ARG;
  }
  const size_t bytes = upf_state_bytes(s);
  if (bytes == 0) {
    set_error("%s: the system has no particles yet", who);
    return UPF_ERR_STATE;
  }
  StateFileHeader h{};
  std::memcpy(h.magic, kStateMagic, 8);
  h.version = kStateVersion;
  h.abi_version = (uint32_t)upf_abi_version();
  h.header_bytes = sizeof(StateFileHeader);
  h.params_bytes = sizeof(upf_params);
  h.state_bytes = bytes;
  upf_params prm{};
  upf_status st = upf_get_params(s, &prm);
  if (st == UPF_OK) st = system_counts(s, &h.n_dynamic, &h.num_bodies);
  if (st != UPF_OK) return st;
  h.method = prm.method;
  std::vector<char> state(bytes);
  if ((st = upf_state_save(s, state.data(), bytes)) != UPF_OK) return st;
  h.checksum = fnv1a(state.data(), bytes, fnv1a(&prm, sizeof prm));
  FILE* f = std::fopen(path, "wb");
  if (!f) {
    set_error("%s: cannot open %s for writing: %s", who, path, std::strerror(errno));
    return UPF_ERR_IO;
  }
  bool ok = std::fwrite(&h, sizeof h, 1, f) == 1 && std::fwrite(&prm, sizeof prm, 1, f) == 1 &&
            std::fwrite(state.data(), 1, bytes, f) == bytes;
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) {
    set_error("%s: writing %s failed: %s", who, path, std::strerror(errno));
    return UPF_ERR_IO;
  }
  return UPF_OK;
}

upf_status upf_state_file_info(const char* path, upf_params* params, uint32_t* n_dynamic, uint32_t* num_bodies,
                               uint64_t* state_bytes) {
  const char* who = "upf_state_file_info";
  if (!path) {
    set_error("%s: null path", who);
    return UPF_ERR_INVALID_ARG;
  }
  FILE* f = std::fopen(path, "rb");
  if (!f) {
    set_error("%s: cannot open %s: %s", who, path, std::strerror(errno));
    return UPF_ERR_IO;
  }
  StateFileHeader h{};
  upf_params prm{};
  const upf_status st = read_header(f, path, h, prm, who);
  std::fclose(f);
  if (st != UPF_OK) return st;
  if (params) *params = prm;
  if (n_dynamic) *n_dynamic = h.n_dynamic;
  if (num_bodies) *num_bodies = h.num_bodies;
  if (state_bytes) *state_bytes = h.state_bytes;
  return UPF_OK;
}

// The name of the first parameter whose stored bits differ between a and b
// (the reserved words are not compared), or null if they all match.
static const char* first_param_difference(const upf_params& a, const upf_params& b) {
  static const struct {
    size_t off, size;
    const char* name;
  } fields[] = {
#define UPF_FIELD(f) {offsetof(upf_params, f), sizeof(((upf_params*)nullptr)->f), #f}
      UPF_FIELD(method), UPF_FIELD(flags), UPF_FIELD(particle_spacing), UPF_FIELD(particle_radius),
      UPF_FIELD(support_radius), UPF_FIELD(mass), UPF_FIELD(rest_density), UPF_FIELD(gas_constant),
      UPF_FIELD(gamma), UPF_FIELD(viscosity), UPF_FIELD(gravity), UPF_FIELD(dt), UPF_FIELD(density_error_factor),
      UPF_FIELD(density_error_fudge), UPF_FIELD(max_density_error), UPF_FIELD(min_loops), UPF_FIELD(max_loops),
      UPF_FIELD(surface_tension_gamma), UPF_FIELD(surface_adhesion_beta), UPF_FIELD(force_distance),
      UPF_FIELD(max_boundary_force), UPF_FIELD(spring_coefficient), UPF_FIELD(spring_coefficient_boundary),
      UPF_FIELD(damping_coefficient), UPF_FIELD(terminal_speed), UPF_FIELD(granular_kr), UPF_FIELD(granular_kd),
      UPF_FIELD(granular_kt), UPF_FIELD(granular_mu), UPF_FIELD(zindex_origin), UPF_FIELD(zindex_extent),
      UPF_FIELD(scales), UPF_FIELD(block_size), UPF_FIELD(collision_min), UPF_FIELD(collision_max),
      UPF_FIELD(container_min), UPF_FIELD(container_max), UPF_FIELD(max_neighbors), UPF_FIELD(search_cell),
#undef UPF_FIELD
  };
  const char* pa = reinterpret_cast<const char*>(&a);
  const char* pb = reinterpret_cast<const char*>(&b);
  for (const auto& f : fields)
    if (std::memcmp(pa + f.off, pb + f.off, f.size) != 0) return f.name;
  return nullptr;
}

upf_status upf_state_read_file(upf_system* s, const char* path) {
  const char* who = "upf_state_read_file";
  if (!s || !path) {
    set_error("%s: null argument", who);
    return UPF_ERR_INVALID_ARG;
  }
  const size_t bytes = upf_state_bytes(s);
  if (bytes == 0) {
    set_error("%s: set the system's particles (the same scene as the saving system's) first", who);
    return UPF_ERR_STATE;
  }
  upf_params mine{};
  uint32_t n_dyn = 0, bodies = 0;
  upf_status st = upf_get_params(s, &mine);
  if (st == UPF_OK) st = system_counts(s, &n_dyn, &bodies);
  if (st != UPF_OK) return st;
  FILE* f = std::fopen(path, "rb");
  if (!f) {
    set_error("%s: cannot open %s: %s", who, path, std::strerror(errno));
    return UPF_ERR_IO;
  }
  StateFileHeader h{};
  upf_params prm{};
  if ((st = read_header(f, path, h, prm, who)) != UPF_OK) {
    std::fclose(f);
    return st;
  }
  if (h.state_bytes != bytes || h.n_dynamic != n_dyn || h.num_bodies != bodies || h.method != mine.method) {
    std::fclose(f);
    set_error("%s: %s holds %u dynamic particles, %u rigid bodies, method %d (%llu B); this system has %u, %u, %d (%zu B)",
              who, path, h.n_dynamic, h.num_bodies, h.method, (unsigned long long)h.state_bytes, n_dyn, bodies,
              mine.method, bytes);
    return UPF_ERR_INVALID_ARG;
  }
  std::vector<char> state(bytes);
  const bool got = std::fread(state.data(), 1, bytes, f) == bytes;
  std::fclose(f);
  if (!got) {
    set_error("%s: %s is truncated", who, path);
    return UPF_ERR_IO;
  }
  if (fnv1a(state.data(), bytes, fnv1a(&prm, sizeof prm)) != h.checksum) {
    set_error("%s: %s fails its checksum (corrupted)", who, path);
    return UPF_ERR_IO;
  }
  // a snapshot resumes only under the physics it was saved with: every
  // parameter word up to the reserved tail must match the system's own
  const char* field = first_param_difference(prm, mine);
  if (field) {
    set_error("%s: %s was saved with different parameters (%s differs); create the system with the file's "
              "parameters (upf_state_file_info returns them)", who, path, field);
    return UPF_ERR_INVALID_ARG;
  }
  return upf_state_load(s, state.data(), bytes);
}
