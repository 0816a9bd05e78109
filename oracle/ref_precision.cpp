// ref_precision.cpp -- TEST INFRASTRUCTURE.  Linked into the oracle/_ref builds of the
// unmodified reference CLI so that every number it prints to stdout (macro strain,
// checkpoint errors, P/Y, tau/Y, effective moduli: EffPlast2D.cu:360, :415, :632-639,
// EffPlast2D.h:124-133) carries 17 significant digits instead of the default 6.
// EffPlast2D.log keeps the reference's own 6-digit formatting.
#include <iostream>

namespace {
struct FullPrecisionCout {
  FullPrecisionCout() { std::cout.precision(17); }
} full_precision_cout;
}  // namespace
