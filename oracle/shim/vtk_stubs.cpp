// Link-time stand-ins for the reference's VTK-backed reader/writer classes.
// VTK is not installed here; oracle decks switch VTU output off and read
// CSV meshes, so none of these is reached.  Each aborts loudly if it is.
// ORACLE TEST INFRASTRUCTURE ONLY.
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>
#include "rw/vtkReader.h"
#include "rw/vtkParticleReader.h"
#include "rw/vtkParticleWriter.h"

namespace {
[[noreturn]] void noVtk(const char *what) {
  std::fprintf(stderr, "peridem_ref: %s needs VTK, which this oracle build does not have\n", what);
  std::abort();
}
}  // namespace

namespace rw {
namespace reader {
VtkReader::VtkReader(const std::string &) { noVtk("VtkReader"); }
void VtkReader::close() { noVtk("VtkReader::close"); }
void VtkReader::readNodes(std::vector<util::Point> *) { noVtk("VtkReader::readNodes"); }
void VtkReader::readMesh(size_t, std::vector<util::Point> *, size_t &, size_t &,
                         std::vector<size_t> *, std::vector<std::vector<size_t>> *,
                         std::vector<double> *, bool) { noVtk("VtkReader::readMesh"); }
void VtkReader::readCells(size_t, size_t &, size_t &, std::vector<size_t> *,
                          std::vector<std::vector<size_t>> *) { noVtk("VtkReader::readCells"); }
bool VtkReader::readPointData(const std::string &, std::vector<uint8_t> *) { noVtk("readPointData"); }
bool VtkReader::readPointData(const std::string &, std::vector<size_t> *) { noVtk("readPointData"); }
bool VtkReader::readPointData(const std::string &, std::vector<int> *) { noVtk("readPointData"); }
bool VtkReader::readPointData(const std::string &, std::vector<float> *) { noVtk("readPointData"); }
bool VtkReader::readPointData(const std::string &, std::vector<double> *) { noVtk("readPointData"); }
bool VtkReader::readPointData(const std::string &, std::vector<util::Point> *) { noVtk("readPointData"); }
bool VtkReader::readPointData(const std::string &, std::vector<util::SymMatrix3> *) { noVtk("readPointData"); }
bool VtkReader::readPointData(const std::string &, std::vector<util::Matrix3> *) { noVtk("readPointData"); }
bool VtkReader::readCellData(const std::string &, std::vector<float> *) { noVtk("readCellData"); }
bool VtkReader::readCellData(const std::string &, std::vector<double> *) { noVtk("readCellData"); }
bool VtkReader::readCellData(const std::string &, std::vector<util::Point> *) { noVtk("readCellData"); }
bool VtkReader::readCellData(const std::string &, std::vector<util::SymMatrix3> *) { noVtk("readCellData"); }
bool VtkReader::readCellData(const std::string &, std::vector<util::Matrix3> *) { noVtk("readCellData"); }
VtkParticleReader::VtkParticleReader(const std::string &) { noVtk("VtkParticleReader"); }
void VtkParticleReader::readNodes(model::ModelData *) { noVtk("VtkParticleReader::readNodes"); }
}  // namespace reader
namespace writer {
VtkParticleWriter::VtkParticleWriter(const std::string &, const std::string &) { noVtk("VtkParticleWriter"); }
void VtkParticleWriter::addTimeStep(const double &) { noVtk("addTimeStep"); }
void VtkParticleWriter::appendMesh(const model::ModelData *, const std::vector<std::string> &) { noVtk("appendMesh"); }
void VtkParticleWriter::appendNodes(const model::ModelData *, const std::vector<std::string> &) { noVtk("appendNodes"); }
void VtkParticleWriter::appendStrainStress(const model::ModelData *) { noVtk("appendStrainStress"); }
void VtkParticleWriter::close() { noVtk("VtkParticleWriter::close"); }
}  // namespace writer
}  // namespace rw
