/*
 * C entry points over the reference's host-side point code compiled here.
 *
 * Test infrastructure only (built into oracle/_ref/, never linked by the
 * product). Each function runs the reference's own routine:
 *   ref_make_points  -> Application::makePoints  Main/Application.cpp:316-473
 *                       with DtRandom            Common/DtRandom.cpp:44-109
 *   ref_read_points  -> Application::readPoints  Main/Application.cpp:475-587
 *   ref_scale_value  -> Application::_scalePoint Main/Application.cpp:589-603
 *   ref_morton_keys  -> GetMortonNumber          GDelaunay/GDelData.cu:51-87
 * The oracle Makefile cuts those function bodies out of the reference files
 * at build time (sed, into oracle/_ref/, never committed) and compiles them
 * against the small stand-ins below for the class and types they use;
 * Config.h, DtRandom.h and DtRandom.cpp are compiled as they are. Point3 is
 * the REAL_TYPE_DOUBLE layout (Common/Geometry.h:53-69), or with
 * REF_REAL_FLOAT defined the default float build's (RealType = float), whose
 * file scaling runs in float arithmetic.
 */
#include "Config.h"
#include "DtRandom.h"

#include <algorithm>
#include <cassert>

#ifdef REF_REAL_FLOAT
typedef float RealType;
#else
typedef double RealType;
#endif

struct Point3 {
    RealType _p[3];
    bool operator<(const Point3& q) const { return std::lexicographical_compare(_p, _p + 3, q._p, q._p + 3); }
};
typedef std::vector<Point3> Point3HVec;
typedef std::set<Point3> Point3Set;

static Config g_config;
Config& getConfig() { return g_config; }

class Application {
public:
    Point3HVec _pointVec;
    Point3HVec _scaledVec;
    void makePoints();
    void readPoints();
    RealType _scalePoint(RealType gridWidth, float minVal, float maxVal, RealType inVal);
};

#include "refapp_extract.inc"

// the Morton functor is device code in the reference; here it runs on the host
#define __device__
#define CudaAssert(x) assert(x)
#include "refmorton_extract.inc"
#undef __device__

static void reset_config(int n, int dist, int grid, int seed) {
    g_config = Config();
    g_config._seed = seed;
    g_config._runNum = 1;
    g_config._gridSize = grid;
    g_config._pointNum = n;
    g_config._dist = (Distribution)dist;
    g_config._logVerbose = false;
    g_config._logStats = false;
    g_config._inFile = false;
}

extern "C" {

int ref_make_points(int n, int dist, int grid, int seed, double* out) {
    reset_config(n, dist, grid, seed);
    Application app;
    app.makePoints();
    for (size_t i = 0; i < app._pointVec.size(); ++i)
        for (int k = 0; k < 3; ++k) out[3 * i + k] = app._pointVec[i]._p[k];
    return (int)app._pointVec.size();
}

// points of the file after readPoints: the scaled unique points (_scaledVec),
// at most cap of them; returns their count
int ref_read_points(const char* path, int grid, double* scaled, int cap) {
    reset_config(0, 0, grid, 0);
    g_config._inFile = true;
    g_config._inFilename = path;
    Application app;
    app.readPoints();
    const int m = (int)app._scaledVec.size();
    for (int i = 0; i < m && i < cap; ++i)
        for (int k = 0; k < 3; ++k) scaled[3 * (size_t)i + k] = app._scaledVec[i]._p[k];
    return m;
}

double ref_scale_value(double grid, float min_val, float max_val, double v) {
    Application app;
    return app._scalePoint(grid, min_val, max_val, v);
}

void ref_morton_keys(const double* pts, int n, int* keys) {
    GetMortonNumber f;
    for (int i = 0; i < n; ++i) {
        Point3 p;
        for (int k = 0; k < 3; ++k) p._p[k] = (RealType)pts[3 * (size_t)i + k];
        keys[i] = f(p);
    }
}

}  // extern "C"
