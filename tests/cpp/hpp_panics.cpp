// Host-side checks of the C++ mirror (no GPU needed): each reference panic
// surfaces as imageproc_b200::Panic with the reference's message.
#include <cstdio>
#include <string>

#include "imageproc_b200/template_matching.hpp"

using namespace imageproc_b200;

static int expect_panic(const char* what, const std::string& msg, void (*fn)()) {
  try {
    fn();
  } catch (const Panic& p) {
    if (msg == p.what()) return 0;
    std::printf("%s: wrong message '%s'\n", what, p.what());
    return 1;
  } catch (...) {
    std::printf("%s: wrong exception type\n", what);
    return 1;
  }
  std::printf("%s: no panic\n", what);
  return 1;
}

int main() {
  int bad = 0;
  bad += expect_panic("width", "image width must be greater than or equal to template width", [] {
    match_template(GrayImage(5, 5), GrayImage(6, 5), MatchTemplateMethod::SumOfSquaredErrors);
  });
  bad += expect_panic("height", "image height must be greater than or equal to template height", [] {
    match_template_parallel(GrayImage(5, 5), GrayImage(5, 6), MatchTemplateMethod::CrossCorrelation);
  });
  bad += expect_panic("mask", "the template and mask must be the same size", [] {
    match_template_with_mask(GrayImage(5, 5), GrayImage(6, 5), MatchTemplateMethod::CrossCorrelation,
                             GrayImage(5, 5));
  });
  bad += expect_panic("empty", "image must be non-empty", [] { find_extremes(Image<float>(0, 4)); });
  if (!bad) std::printf("ok\n");
  return bad;
}
