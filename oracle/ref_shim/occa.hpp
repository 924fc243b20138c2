// Host-only stand-in for the OCCA API surface that the reference's host code
// uses (include/utils.hpp:37-45, include/memory.hpp:287-698,
// include/platform.hpp:61-185).  TEST INFRASTRUCTURE: it lets the reference's
// own mesh, ogs and primitives sources compile and run on the CPU so that their
// outputs can pin the oracle; it is never linked into the product.
//
// "Device" memory is host memory, so the reference's host-side setup and its
// copies run unchanged.  Kernels are never run: calling one throws, naming
// the kernel, so an unexpected device call cannot pass silently.
#pragma once

// the real OCCA header brings these standard headers with it; the reference relies on that
#include <cstddef>
#include <cstdint>
#include <cstring>
#include <functional>
#include <iostream>
#include <map>
#include <sstream>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

namespace occa {

// A JSON-like property tree: a scalar (kept as text) or an object of named
// children.  Only what the reference assigns and reads is supported.
class json {
 public:
  json() = default;
  json(bool v) : value_(v ? "true" : "false") {}
  json(int v) : value_(std::to_string(v)) {}
  json(long v) : value_(std::to_string(v)) {}
  json(long long v) : value_(std::to_string(v)) {}
  json(unsigned v) : value_(std::to_string(v)) {}
  json(unsigned long v) : value_(std::to_string(v)) {}
  json(float v) : value_(std::to_string(v)) {}
  json(double v) : value_(std::to_string(v)) {}
  json(const char* v) : value_(v) {}
  json(const std::string& v) : value_(v) {}
  json(const std::string& key, const json& value) { (*this)[key] = value; }   // a one-entry object

  json& operator[](const std::string& key) {
    if (!children_) children_ = std::make_shared<std::map<std::string, json>>();
    return (*children_)[key];
  }
  json& operator+=(const std::string& s) {
    value_ += s;
    return *this;
  }
  bool has(const std::string& key) const { return children_ && children_->count(key); }
  std::string toString() const { return value_; }
  template <class T>
  T get(const std::string& key, const T& def = T()) const {
    (void)key;
    return def;
  }

 private:
  std::string value_;
  std::shared_ptr<std::map<std::string, json>> children_;
};
using properties = json;

struct dtype_t {
  size_t bytes = 1;
};
namespace dtype {
template <class T>
inline dtype_t get() {
  return dtype_t{sizeof(T)};
}
}  // namespace dtype

class stream {
 public:
  stream() = default;
  bool isInitialized() const { return false; }
};

class memory {
 public:
  memory() = default;
  memory(std::shared_ptr<char> base, size_t offset, size_t bytes) : base_(base), offset_(offset), bytes_(bytes) {}

  bool isInitialized() const { return base_ != nullptr; }
  void setDtype(const dtype_t& d) { dtype_bytes_ = d.bytes; }
  void* ptr() { return base_ ? base_.get() + offset_ : nullptr; }
  const void* ptr() const { return base_ ? base_.get() + offset_ : nullptr; }
  size_t size() const { return bytes_; }
  size_t length() const { return dtype_bytes_ ? bytes_ / dtype_bytes_ : bytes_; }

  memory operator+(ptrdiff_t offset) const { return slice(offset); }
  memory slice(ptrdiff_t offset, ptrdiff_t count = -1) const {
    const size_t off = (size_t)offset * dtype_bytes_;
    if (off > bytes_) throw std::runtime_error("occa shim: memory slice beyond the allocation");
    const size_t n = count < 0 ? bytes_ - off : (size_t)count * dtype_bytes_;
    memory m(base_, offset_ + off, n);
    m.dtype_bytes_ = dtype_bytes_;
    return m;
  }

  void copyFrom(const void* src, size_t bytes, size_t offset = 0, const json& = json()) {
    check(offset, bytes);
    if (bytes) std::memcpy(static_cast<char*>(ptr()) + offset, src, bytes);
  }
  void copyFrom(const memory& src, size_t bytes, size_t destOffset = 0, size_t srcOffset = 0,
                const json& = json()) {
    check(destOffset, bytes);
    src.check(srcOffset, bytes);
    if (bytes) std::memmove(static_cast<char*>(ptr()) + destOffset, static_cast<const char*>(src.ptr()) + srcOffset,
                            bytes);
  }
  void copyTo(void* dest, size_t bytes, size_t offset = 0, const json& = json()) const {
    check(offset, bytes);
    if (bytes) std::memcpy(dest, static_cast<const char*>(ptr()) + offset, bytes);
  }
  void copyTo(memory dest, size_t bytes, size_t destOffset = 0, size_t srcOffset = 0, const json& = json()) const {
    dest.copyFrom(*this, bytes, destOffset, srcOffset);
  }
  void swap(memory& m) { std::swap(*this, m); }
  void free() {
    base_.reset();
    bytes_ = offset_ = 0;
  }

 private:
  void check(size_t offset, size_t bytes) const {
    if (offset + bytes > bytes_) throw std::runtime_error("occa shim: copy beyond the allocation");
  }
  std::shared_ptr<char> base_;
  size_t offset_ = 0, bytes_ = 0, dtype_bytes_ = 1;
};

class kernel {
 public:
  kernel() = default;
  explicit kernel(const std::string& name) : name_(name) {}
  bool isInitialized() const { return !name_.empty(); }
  template <class... A>
  void operator()(A&&...) const {
    throw std::runtime_error("occa shim: device kernel '" + name_ +
                             "' called in the host-only build of the reference (no device code runs here)");
  }

 private:
  std::string name_;
};

class device {
 public:
  device() = default;
  explicit device(const json&) : init_(true) {}
  bool isInitialized() const { return init_; }
  std::string mode() const { return "Serial"; }
  memory malloc(size_t bytes, const void* src = nullptr, const json& = json()) {
    std::shared_ptr<char> p(new char[bytes ? bytes : 1](), std::default_delete<char[]>());
    if (src && bytes) std::memcpy(p.get(), src, bytes);
    return memory(p, 0, bytes);
  }
  template <class T>
  memory malloc(size_t count, const void* src = nullptr, const json& props = json()) {
    memory m = malloc(count * sizeof(T), src, props);
    m.setDtype(dtype::get<T>());
    return m;
  }
  template <class T>
  memory malloc(size_t count, const json& props) {
    return malloc<T>(count, nullptr, props);
  }
  void finish() {}
  stream getStream() { return stream(); }
  void setStream(const stream&) {}
  stream createStream() { return stream(); }

 private:
  bool init_ = false;
};

inline int getDeviceCount(const std::string&) { return 1; }
namespace env {
inline void setOccaCacheDir(const std::string&) {}
}  // namespace env

}  // namespace occa
