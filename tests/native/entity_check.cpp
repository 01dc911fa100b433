// Host build of the 2D boundary-entity geometry (egg_b200/csrc/entity2.cuh):
// reads lines "tag p0 .. p9 g0 g1 h00 h01 h10 h11 x y" from stdin and
// prints "step_x step_y foot_x foot_y" for each, so the tests can compare the
// Newton step and the projection with the reference core's own.
#include <cmath>
#include <cstdio>

#include "entity2.cuh"

using namespace egg_b200;

int main()
{
    int tag;
    double e[10], g[2], h[4], x, y;
    while (std::scanf("%d", &tag) == 1) {
        for (double& v : e) { std::scanf("%lf", &v); }
        if (std::scanf("%lf %lf %lf %lf %lf %lf %lf %lf", &g[0], &g[1], &h[0], &h[1], &h[2], &h[3], &x, &y) != 8) {
            return 1;
        }
        double st[2], fx, fy;
        entity_newton_step(tag, e, h, g, x, y, st);
        entity_project(tag, e, x, y, fx, fy);
        std::printf("%.17g %.17g %.17g %.17g\n", st[0], st[1], fx, fy);
    }
    return 0;
}
