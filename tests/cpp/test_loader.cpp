// Problem-file readers of include/nelson_b200/nelson.hpp (no GPU needed):
// writes small synthetic files, reads them back, checks the values and that
// truncated files and out-of-range indices are rejected.
#include <cstdio>
#include <fstream>
#include <string>

#include "nelson_b200/nelson.hpp"

static int failures = 0;
static void expect(bool ok, const char* what) {
  std::printf("%s %s\n", ok ? "ok  " : "FAIL", what);
  if (!ok) failures++;
}

int main(int argc, char** argv) {
  const std::string dir = argc > 1 ? argv[1] : ".";
  {
    std::ofstream f(dir + "/vis.txt");
    f << "3 5 4\n0 0\n1 0\n2 4\n0 3\n";
  }
  nelson_b200::Problem p;
  expect(p.load(dir + "/vis.txt"), "visibility list loads");
  expect(p.nCameras == 3 && p.nPoints == 5 && p.edges.size() == 4, "visibility list sizes");
  expect(p.edges[2].first == 2 && p.edges[2].second == 4, "visibility list pair");
  {
    std::ofstream f(dir + "/vis_bad.txt");
    f << "3 5 2\n0 0\n3 1\n";
  }
  expect(!p.load(dir + "/vis_bad.txt"), "out-of-range camera rejected");
  expect(!p.load(dir + "/missing.txt"), "missing file rejected");
  {
    std::ofstream f(dir + "/p.bal");
    f << "1 2 2\n0 0 -1.5 2.5\n0 1 3.0 -4.0\n";
    for (int i = 0; i < 9; i++) f << 0.1 * i << "\n";
    for (int i = 0; i < 6; i++) f << 1.0 + i << "\n";
  }
  nelson_b200::BALData b;
  expect(b.load(dir + "/p.bal"), "BAL loads");
  expect(b.nCameras == 1 && b.nPoints == 2 && b.cam.size() == 2, "BAL sizes");
  expect(b.obs[0] == -1.5 && b.obs[3] == -4.0 && b.cams[8] == 0.8 && b.pts[5] == 6.0, "BAL values");
  {
    std::ofstream f(dir + "/short.bal");
    f << "1 2 2\n0 0 -1.5 2.5\n";
  }
  expect(!b.load(dir + "/short.bal"), "truncated BAL rejected");
  std::printf(failures ? "FAILED %d\n" : "ALL OK\n", failures);
  return failures ? 1 : 0;
}
