// template_matching.hpp -- C++ host API mirroring imageproc::template_matching.
//
// Header-only layer over the C ABI (imageproc_b200.h). Same function names and
// argument meaning as imageproc 0.27.0 src/template_matching.rs; where the
// reference panics, these functions throw imageproc_b200::Panic carrying the
// reference's assertion message. Device failures throw DeviceError.
#pragma once

#include <cstdint>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "imageproc_b200.h"

namespace imageproc_b200 {

// A single-channel image, row-major, stride == width (the reference's Image<P>).
template <typename T>
struct Image {
  uint32_t width = 0, height = 0;
  std::vector<T> data;
  Image() = default;
  Image(uint32_t w, uint32_t h) : width(w), height(h), data(size_t(w) * h) {}
  T& at(uint32_t x, uint32_t y) { return data[size_t(y) * width + x]; }
  const T& at(uint32_t x, uint32_t y) const { return data[size_t(y) * width + x]; }
};
using GrayImage = Image<uint8_t>;

enum class MatchTemplateMethod : int {
  SumOfSquaredErrors = IPB_SUM_OF_SQUARED_ERRORS,
  SumOfSquaredErrorsNormalized = IPB_SUM_OF_SQUARED_ERRORS_NORMALIZED,
  CrossCorrelation = IPB_CROSS_CORRELATION,
  CrossCorrelationNormalized = IPB_CROSS_CORRELATION_NORMALIZED,
};

struct Panic : std::logic_error {
  using std::logic_error::logic_error;
};
struct DeviceError : std::runtime_error {
  using std::runtime_error::runtime_error;
};

inline void check(ipb_status st) {
  if (st == IPB_OK) return;
  const std::string msg = ipb_last_error_message();
  if (st == IPB_ERR_TEMPLATE_WIDTH || st == IPB_ERR_TEMPLATE_HEIGHT || st == IPB_ERR_MASK_SIZE ||
      st == IPB_ERR_EMPTY_IMAGE)
    throw Panic(msg);
  if (st == IPB_ERR_INVALID_ARGUMENT) throw std::invalid_argument(msg);
  throw DeviceError(msg);
}

namespace detail {
inline Image<float> output_for(const GrayImage& image, const GrayImage& templ) {
  if (image.width < templ.width || image.height < templ.height) return Image<float>();
  return Image<float>(image.width - templ.width + 1, image.height - templ.height + 1);
}
}  // namespace detail

// match_template (src/template_matching.rs:78-92)
inline Image<float> match_template(const GrayImage& image, const GrayImage& templ,
                                   MatchTemplateMethod method) {
  Image<float> out = detail::output_for(image, templ);
  check(ipb_match_template(image.data.data(), image.width, image.height, templ.data.data(),
                           templ.width, templ.height, int(method), out.data.data()));
  return out;
}

// match_template_parallel (src/template_matching.rs:96-110)
inline Image<float> match_template_parallel(const GrayImage& image, const GrayImage& templ,
                                            MatchTemplateMethod method) {
  Image<float> out = detail::output_for(image, templ);
  check(ipb_match_template_parallel(image.data.data(), image.width, image.height,
                                    templ.data.data(), templ.width, templ.height, int(method),
                                    out.data.data()));
  return out;
}

// match_template_with_mask (src/template_matching.rs:125-140)
inline Image<float> match_template_with_mask(const GrayImage& image, const GrayImage& templ,
                                             MatchTemplateMethod method, const GrayImage& mask) {
  Image<float> out = detail::output_for(image, templ);
  check(ipb_match_template_with_mask(image.data.data(), image.width, image.height,
                                     templ.data.data(), templ.width, templ.height, int(method),
                                     mask.data.data(), mask.width, mask.height, out.data.data()));
  return out;
}

// match_template_with_mask_parallel (src/template_matching.rs:144-163)
inline Image<float> match_template_with_mask_parallel(const GrayImage& image,
                                                      const GrayImage& templ,
                                                      MatchTemplateMethod method,
                                                      const GrayImage& mask) {
  Image<float> out = detail::output_for(image, templ);
  check(ipb_match_template_with_mask_parallel(
      image.data.data(), image.width, image.height, templ.data.data(), templ.width, templ.height,
      int(method), mask.data.data(), mask.width, mask.height, out.data.data()));
  return out;
}

// Extremes<T> (src/template_matching.rs:466-475)
template <typename T>
struct Extremes {
  T max_value;
  T min_value;
  std::pair<uint32_t, uint32_t> max_value_location;
  std::pair<uint32_t, uint32_t> min_value_location;
  bool operator==(const Extremes& o) const {
    return max_value == o.max_value && min_value == o.min_value &&
           max_value_location == o.max_value_location && min_value_location == o.min_value_location;
  }
};

namespace detail {
#define IPB_CPP_EXTREMES(T, S)                                                             \
  inline ipb_status find_extremes_c(const Image<T>& im, Extremes<T>& out) {              \
    ipb_extremes_##S r{};                                                                \
    ipb_status st = ipb_find_extremes_##S(im.data.data(), im.width, im.height, &r);      \
    out = Extremes<T>{r.max_value, r.min_value,                                          \
                      {r.max_value_location_x, r.max_value_location_y},                  \
                      {r.min_value_location_x, r.min_value_location_y}};                 \
    return st;                                                                           \
  }
IPB_CPP_EXTREMES(uint8_t, u8)
IPB_CPP_EXTREMES(uint16_t, u16)
IPB_CPP_EXTREMES(uint32_t, u32)
IPB_CPP_EXTREMES(uint64_t, u64)
IPB_CPP_EXTREMES(int8_t, i8)
IPB_CPP_EXTREMES(int16_t, i16)
IPB_CPP_EXTREMES(int32_t, i32)
IPB_CPP_EXTREMES(int64_t, i64)
IPB_CPP_EXTREMES(float, f32)
IPB_CPP_EXTREMES(double, f64)
#undef IPB_CPP_EXTREMES
}  // namespace detail

// find_extremes<T> (src/template_matching.rs:479-511)
template <typename T>
inline Extremes<T> find_extremes(const Image<T>& image) {
  Extremes<T> out{};
  check(detail::find_extremes_c(image, out));
  return out;
}

}  // namespace imageproc_b200
