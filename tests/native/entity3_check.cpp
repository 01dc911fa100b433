// Host build of the 3D boundary-entity projection (egg_b200/csrc/entity3.cuh):
// reads lines "tag p0 .. p9 x y z" from stdin and prints the foot "fx fy fz",
// so the tests can compare it with the reference core's own projection.
#include <cmath>
#include <cstdio>

#include "entity3.cuh"

using namespace egg_b200;

int main()
{
    int tag;
    double e[10], p[3], f[3];
    while (std::scanf("%d", &tag) == 1) {
        for (double& v : e) { std::scanf("%lf", &v); }
        if (std::scanf("%lf %lf %lf", &p[0], &p[1], &p[2]) != 3) { return 1; }
        entity3_project(tag, e, p, f);
        std::printf("%.17g %.17g %.17g\n", f[0], f[1], f[2]);
    }
    return 0;
}
