// The parts of the reference library that its SceneBase (the camera store
// every backend shares) needs, compiled from the reference's own sources in
// the order its unity build (src/Ray/_Ray.cpp) compiles them, without the
// factory and the backends: SceneBase.cpp and the core it calls
// (ConstructCamera, internal/Core.cpp, with internal/BVHSplit.cpp before it).
// The standard headers first: the unity build has them from the files before.
#include <algorithm>
#include <cassert>
#include <cfloat>
#include <climits>
#include <cmath>
#include <cstring>
#include <limits>
#include <memory>
#include <vector>

#include "Ray/SceneBase.cpp"
#include "Ray/internal/BVHSplit.cpp"
#include "Ray/internal/Core.cpp"
