// Host side of the VTK output (clover_visit.cu): one frame is the host copy
// of every chunk's fields at one step, written by write_visit_frame.
#pragma once

#include <string>
#include <vector>

namespace clover {

struct VisitChunk {
  int chunk;       // chunk number in the file names (1 for a single chunk)
  int nx, ny, nz;  // cells
  // reference layouts, FP64: cell arrays (n+4)^3 and node arrays (n+5)^3
  // from min-2, vertex coordinates from min (n+1 values)
  std::vector<double> density0, energy0, pressure, viscosity, xvel0, yvel0, zvel0;
  std::vector<double> vertexx, vertexy, vertexz;
};

struct VisitFrame {
  std::string dir;  // output directory
  int step;
  bool first;       // the first frame of the run starts clover.visit
  std::vector<VisitChunk> chunks;
};

void format_e12_4(double v, char out[13]);
bool write_visit_frame(const VisitFrame& fr, std::string* err);

}  // namespace clover
