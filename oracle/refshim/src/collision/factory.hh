// Stand-in for the reference's src/collision/factory.hh inside the reference
// harness build (oracle/ref_harness.cu).  The real header builds shapes with
// Eigen, which is not installed here; the harness never calls the shape
// factory (it constructs shapes with the shapes.hh constructors), and the only
// thing src/batch_cc.cu takes from that header is its global
// `using namespace ppln;`, reproduced below.  Test infrastructure only.
#pragma once
namespace ppln {}
using namespace ppln;
