// Byte-compatible FEMInputs / FEMOutputs codec; see wire.hpp for the layout.
#include "wire.hpp"

#include <cstring>
#include <mutex>
#include <unordered_map>

namespace sgs {

namespace {
constexpr size_t HUGE_PAGE = size_t(2) << 20, HOST_CACHE_BYTES = size_t(4) << 30;
struct HostCache {
  std::mutex mutex;
  std::multimap<size_t, void*> free_blocks;   // size -> released block
  std::unordered_map<void*, size_t> live;     // block handed out -> its size
  size_t cached = 0;                          // bytes in free_blocks
};
// never destroyed: buffers of static objects may be released after exit begins
HostCache& host_cache() {
  static HostCache* c = new HostCache;
  return *c;
}
}  // namespace

void* host_large_alloc(size_t bytes) {
  const size_t rounded = (bytes + HUGE_PAGE - 1) & ~(HUGE_PAGE - 1);
  HostCache& c = host_cache();
  std::lock_guard<std::mutex> lock(c.mutex);
  auto it = c.free_blocks.lower_bound(rounded);
  if (it != c.free_blocks.end() && it->first - rounded <= rounded / 4) {
    void* p = it->second;
    c.cached -= it->first;
    c.live.emplace(p, it->first);
    c.free_blocks.erase(it);
    return p;
  }
  void* p = std::aligned_alloc(HUGE_PAGE, rounded);
  if (!p) {  // give the cached blocks back and try once more
    for (auto& fb : c.free_blocks) std::free(fb.second);
    c.free_blocks.clear();
    c.cached = 0;
    p = std::aligned_alloc(HUGE_PAGE, rounded);
    if (!p) throw std::bad_alloc();
  }
  madvise(p, rounded, MADV_HUGEPAGE);  // advice only; without it the buffer works the same
  c.live.emplace(p, rounded);
  return p;
}

void host_large_free(void* p) {
  if (!p) return;
  HostCache& c = host_cache();
  std::lock_guard<std::mutex> lock(c.mutex);
  auto it = c.live.find(p);
  if (it == c.live.end()) return;  // not a block of this allocator
  const size_t size = it->second;
  c.live.erase(it);
  if (c.cached + size <= HOST_CACHE_BYTES) {
    c.free_blocks.emplace(size, p);
    c.cached += size;
  } else {
    std::free(p);
  }
}

namespace {

// Writes a record into a caller-sized buffer; with no buffer it only counts
// bytes, so an encoder runs once to size its output and once to fill it.
class Writer {
 public:
  explicit Writer(uint8_t* dst = nullptr) : dst_(dst) {}
  void bytes(const void* p, size_t n) {
    if (dst_ && n) std::memcpy(dst_ + pos_, p, n);
    pos_ += n;
  }
  template <typename T>
  void pod(const T& v) { bytes(&v, sizeof(T)); }
  void count(size_t n) { pod<uint64_t>(uint64_t(n)); }
  void str(const std::string& s) {
    count(s.size());
    bytes(s.data(), s.size());
  }
  template <typename V, typename F>
  void map(const std::map<std::string, V>& m, F&& val) {
    count(m.size());
    for (auto& kv : m) {
      str(kv.first);
      val(kv.second);
    }
  }
  // records of {int base[3]; double data[64*width]}, copied block-parallel;
  // with `fill` the payloads come from it instead of g.data
  void grid(const BlockedGrid& g, int width, const GridFill* fill = nullptr) {
    for (int v = 0; v < 3; ++v) pod<int32_t>(g.resolution[v]);
    const size_t n = g.num_blocks(), payload = sizeof(double) * 64 * size_t(width), rec = 12 + payload;
    if (!fill && g.data.size() != n * 64 * size_t(width)) throw WireError("grid payload size mismatch");
    count(n);
    if (dst_) {
      uint8_t* at = dst_ + pos_;
#pragma omp parallel for schedule(static) if (n > 4096)
      for (long b = 0; b < long(n); ++b) {
        std::memcpy(at + size_t(b) * rec, &g.base[3 * size_t(b)], 12);
        if (!fill) std::memcpy(at + size_t(b) * rec + 12, &g.data[size_t(b) * 64 * width], payload);
      }
      if (fill && n) (*fill)(at + 12, rec, n);
    }
    pos_ += n * rec;
  }
  size_t size() const { return pos_; }
  void finish() {
    const uint64_t n = pos_;
    if (dst_) std::memcpy(dst_, &n, 8);
  }

 private:
  uint8_t* dst_;
  size_t pos_ = 8;  // the length header comes first
};

class Reader {
 public:
  explicit Reader(const void* blob) : p_(static_cast<const uint8_t*>(blob)) {
    if (!p_) throw WireError("null blob");
    std::memcpy(&total_, p_, 8);
    if (total_ < 8) throw WireError("length header smaller than the header itself");
    head_ = 8;
  }
  void bytes(void* out, size_t n) {
    if (n > total_ - head_) throw WireError("blob truncated");
    if (n) std::memcpy(out, p_ + head_, n);
    head_ += n;
  }
  template <typename T>
  T pod() {
    T v;
    bytes(&v, sizeof(T));
    return v;
  }
  size_t count(size_t elem_size) {
    uint64_t n = pod<uint64_t>();
    if (elem_size && n > (total_ - head_) / elem_size) throw WireError("element count exceeds blob size");
    return size_t(n);
  }
  std::string str() {
    size_t n = count(1);
    std::string s(n, '\0');
    bytes(&s[0], n);
    return s;
  }
  template <typename V, typename F>
  void map(std::map<std::string, V>& m, F&& val) {
    size_t n = count(8);
    m.clear();
    for (size_t i = 0; i < n; ++i) {
      std::string k = str();
      m[k] = val();
    }
  }
  void grid(BlockedGrid& g, int width) {
    for (int v = 0; v < 3; ++v) g.resolution[v] = pod<int32_t>();
    const size_t rec = 12 + sizeof(double) * 64 * width;
    size_t n = count(rec);
    g.base.resize(n * 3);
    g.data.resize(n * 64 * width);
    const uint8_t* at = p_ + head_;
    const size_t payload = rec - 12;
#pragma omp parallel for schedule(static) if (n > 4096)
    for (long b = 0; b < long(n); ++b) {
      std::memcpy(&g.base[3 * size_t(b)], at + size_t(b) * rec, 12);
      std::memcpy(&g.data[size_t(b) * 64 * width], at + size_t(b) * rec + 12, payload);
    }
    head_ += n * rec;
  }
  void done() const {
    if (head_ != total_) throw WireError("trailing bytes after the record");
  }

 private:
  const uint8_t* p_;
  uint64_t total_ = 0, head_ = 0;
};

void write_base(Writer& w, const FEMBase& b) {
  w.pod(b.version_major);
  w.pod(b.version_minor);
  w.map(b.extra_strings, [&](const std::string& v) { w.str(v); });
  w.map(b.extra_ints, [&](int32_t v) { w.pod(v); });
  w.map(b.extra_doubles, [&](double v) { w.pod(v); });
}

void read_base(Reader& r, FEMBase& b) {
  b.version_major = r.pod<int32_t>();
  b.version_minor = r.pod<int32_t>();
  // fem_interface.h:185-186
  if (b.version_major != 3 || b.version_minor > 1) throw WireError("unsupported interface version");
  r.map(b.extra_strings, [&] { return r.str(); });
  r.map(b.extra_ints, [&] { return r.pod<int32_t>(); });
  r.map(b.extra_doubles, [&] { return r.pod<double>(); });
}

template <typename T>
void write_records(Writer& w, const std::vector<T>& v, size_t rec) {
  w.count(v.size());
  for (auto& x : v) w.bytes(&x, rec);
}

template <typename T>
void read_records(Reader& r, std::vector<T>& v, size_t rec) {
  size_t n = r.count(rec);
  v.resize(n);
  for (auto& x : v) r.bytes(&x, rec);
}

// On-wire sizes: ForceOnNode = int[3] + double[3] = 36, DirichletOnNode = int[3] + int + double = 24
constexpr size_t FORCE_BYTES = 36, DIRICHLET_BYTES = 24;

template <typename T>
void write_packed(Writer& w, const std::vector<T>& v, size_t rec);
template <>
void write_packed(Writer& w, const std::vector<ForceOnNode>& v, size_t) {
  w.count(v.size());
  for (auto& x : v) {
    w.bytes(x.coord, 12);
    w.bytes(x.f, 24);
  }
}
template <>
void write_packed(Writer& w, const std::vector<DirichletOnNode>& v, size_t) {
  w.count(v.size());
  for (auto& x : v) {
    w.bytes(x.coord, 12);
    w.pod(x.axis);
    w.pod(x.value);
  }
}
void read_packed(Reader& r, std::vector<ForceOnNode>& v) {
  size_t n = r.count(FORCE_BYTES);
  v.resize(n);
  for (auto& x : v) {
    r.bytes(x.coord, 12);
    r.bytes(x.f, 24);
  }
}
void read_packed(Reader& r, std::vector<DirichletOnNode>& v) {
  size_t n = r.count(DIRICHLET_BYTES);
  v.resize(n);
  for (auto& x : v) {
    r.bytes(x.coord, 12);
    x.axis = r.pod<int32_t>();
    x.value = r.pod<double>();
  }
}

}  // namespace

FEMInputs decode_inputs(const void* blob) {
  Reader r(blob);
  FEMInputs p;
  read_base(r, p);
  p.dx = r.pod<double>();
  p.preserved_buffer_size = r.pod<uint64_t>();
  p.use_density_only = r.pod<uint8_t>() != 0;
  if (p.use_density_only) {
    p.global_mu = r.pod<double>();
    p.global_lambda = r.pod<double>();
    r.grid(p.density, 1);
  } else {
    r.grid(p.mu, 1);
    r.grid(p.lambda, 1);
  }
  p.mg_level = r.pod<int32_t>();
  p.explicit_mg_level = r.pod<int32_t>();
  p.pre_and_post_smoothing_iter = r.pod<int32_t>();
  p.bottom_smoothing_iter = r.pod<int32_t>();
  p.jacobi_damping = r.pod<double>();
  for (int v = 0; v < 3; ++v) p.resolution[v] = r.pod<int32_t>();
  read_packed(r, p.forces);
  read_packed(r, p.dirichlet_nodes);
  read_packed(r, p.dirichlet_cells);
  p.krylov.tolerance = r.pod<double>();
  p.krylov.max_iterations = r.pod<int32_t>();
  p.krylov.restart_iterations = r.pod<int32_t>();
  p.krylov.print_residuals = r.pod<uint8_t>() != 0;
  p.caller_method = r.str();
  r.done();
  return p;
}

static void write_inputs(Writer& w, const FEMInputs& p) {
  write_base(w, p);
  w.pod(p.dx);
  w.pod(p.preserved_buffer_size);
  w.pod<uint8_t>(p.use_density_only ? 1 : 0);
  if (p.use_density_only) {
    w.pod(p.global_mu);
    w.pod(p.global_lambda);
    w.grid(p.density, 1);
  } else {
    w.grid(p.mu, 1);
    w.grid(p.lambda, 1);
  }
  w.pod(p.mg_level);
  w.pod(p.explicit_mg_level);
  w.pod(p.pre_and_post_smoothing_iter);
  w.pod(p.bottom_smoothing_iter);
  w.pod(p.jacobi_damping);
  for (int v = 0; v < 3; ++v) w.pod(p.resolution[v]);
  write_packed(w, p.forces, 0);
  write_packed(w, p.dirichlet_nodes, 0);
  write_packed(w, p.dirichlet_cells, 0);
  w.pod(p.krylov.tolerance);
  w.pod(p.krylov.max_iterations);
  w.pod(p.krylov.restart_iterations);
  w.pod<uint8_t>(p.krylov.print_residuals ? 1 : 0);
  w.str(p.caller_method);
}

std::vector<uint8_t> encode_inputs(const FEMInputs& p) {
  Writer sizer;
  write_inputs(sizer, p);
  std::vector<uint8_t> out(sizer.size());
  Writer w(out.data());
  write_inputs(w, p);
  w.finish();
  return out;
}

static void write_outputs(Writer& w, const FEMOutputs& o, const GridFill* fill = nullptr) {
  write_base(w, o);
  w.grid(o.displacements, 4, fill);
  w.grid(o.residual_field, 1);
  w.str(o.info);
  w.count(o.residuals.size());
  w.bytes(o.residuals.data(), sizeof(double) * o.residuals.size());
  w.pod(o.error_code);
  w.pod<uint8_t>(o.success ? 1 : 0);
}

char* encode_outputs(const FEMOutputs& o, size_t* length) {
  Writer sizer;
  write_outputs(sizer, o);
  char* out = new char[sizer.size()];
  Writer w(reinterpret_cast<uint8_t*>(out));
  write_outputs(w, o);
  w.finish();
  if (length) *length = sizer.size();
  return out;
}

// Offset of the value of extra_doubles[key] in an encoded FEMOutputs blob: the
// length header, the two version ints, extra_strings and extra_ints, then the
// extra_doubles entries in key order (count, then length-prefixed key and value).
static size_t output_double_offset(const FEMOutputs& o, const std::string& key) {
  size_t pos = 8 + 4 + 4 + 8;
  for (auto& kv : o.extra_strings) pos += 8 + kv.first.size() + 8 + kv.second.size();
  pos += 8;
  for (auto& kv : o.extra_ints) pos += 8 + kv.first.size() + 4;
  pos += 8;
  for (auto& kv : o.extra_doubles) {
    pos += 8 + kv.first.size();
    if (kv.first == key) return pos;
    pos += 8;
  }
  throw WireError("no such output entry: " + key);
}

void patch_output_double(char* blob, const FEMOutputs& o, const std::string& key, double value) {
  std::memcpy(blob + output_double_offset(o, key), &value, sizeof(double));
}

char* encode_outputs(const FEMOutputs& o, size_t* length, const GridFill& fill) {
  return encode_outputs(o, length, fill, nullptr, 0);
}

char* encode_outputs(const FEMOutputs& o, size_t* length, const GridFill& fill, char* buffer, size_t capacity) {
  Writer sizer;
  write_outputs(sizer, o, &fill);
  char* out = buffer;
  if (!out || capacity < sizer.size()) {
    delete[] buffer;
    out = new char[sizer.size()];
  }
  try {
    Writer w(reinterpret_cast<uint8_t*>(out));
    write_outputs(w, o, &fill);
    w.finish();
  } catch (...) {
    delete[] out;
    throw;
  }
  if (length) *length = sizer.size();
  return out;
}

FEMOutputs decode_outputs(const void* blob) {
  Reader r(blob);
  FEMOutputs o;
  read_base(r, o);
  r.grid(o.displacements, 4);
  r.grid(o.residual_field, 1);
  o.info = r.str();
  size_t n = r.count(8);
  o.residuals.resize(n);
  r.bytes(o.residuals.data(), 8 * n);
  o.error_code = r.pod<int32_t>();
  o.success = r.pod<uint8_t>() != 0;
  r.done();
  return o;
}

}  // namespace sgs
