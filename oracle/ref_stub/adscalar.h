// Declaration-only stand-in for A2D's adscalar.h (A2D is not part of the
// reference checkout).  It lets element/LagrangeShapeFuncs.h parse; the only
// user of the type is the generic template for orders above 4, which the
// table dump never instantiates.  No arithmetic lives here.
#pragma once
namespace A2D {
template <typename T, int N>
class ADScalar;
}
