// DataOut without VTK: the reference's result writer interface
// (Explicit3D/include/dataOut.h:44-97) writing VTK XML unstructured-grid files
// (.vtu, ASCII) directly.  The reference builds these files through the VTK
// library (Explicit3D/source/dataOut.cpp), which the GPU drop-in does not
// link; the written file carries the same mesh, node fields and element
// fields: points, hexahedra (VTK cell type 12) with the reference's local node
// order, which is VTK's, one PointData array per add_node_data call and one
// CellData array per add_ele_data call (scalar: 1 component, vector: 3,
// symmetric tensor: 6), and the time as FieldData "TimeValue".
// write_vtu_virtualParticles writes nothing: there are no FSI particles.
#include "dataOut.h"

#include <cstdio>
#include <stdexcept>

namespace EnSC {

DataOut::DataOut(const Types::VerticesAll<3>& pVerticesAll, const std::vector<Element_HexN8>& pTriaHex,
                 Types::Real t)
    : opVerticesAll(pVerticesAll), opTriaHex(pTriaHex), time(t) {}

void DataOut::add_node_data(DataOutType::DataType dataType, const Eigen::Matrix<Types::Real, Eigen::Dynamic, 1>* vec,
                            std::string name) {
    opDataType.push_back(dataType);
    opVec.push_back(vec);
    opName.push_back(name);
}

void DataOut::add_ele_data(DataOutType::DataType dataType, const Eigen::Matrix<Types::Real, Eigen::Dynamic, 1>* vec,
                           std::string name) {
    opDataType_Ele.push_back(dataType);
    opVec_Ele.push_back(vec);
    opName_Ele.push_back(name);
}

namespace {

int components(DataOutType::DataType t) {
    switch (t) {
        case DataOutType::scalar: return 1;
        case DataOutType::vector: return 3;
        default: return 6;
    }
}

void write_array(FILE* f, const std::string& name, int comps, const Eigen::Matrix<Types::Real, Eigen::Dynamic, 1>* v,
                 std::size_t n_items) {
    std::fprintf(f, "<DataArray type=\"Float64\" Name=\"%s\" NumberOfComponents=\"%d\" format=\"ascii\">\n",
                 name.c_str(), comps);
    const std::size_t want = n_items * static_cast<std::size_t>(comps);
    const std::size_t have = v ? static_cast<std::size_t>(v->size()) : 0;
    for (std::size_t i = 0; i < want; ++i)
        std::fprintf(f, "%.17g%c", i < have ? (*v)[static_cast<Eigen::Index>(i)] : 0.0,
                     (i + 1) % static_cast<std::size_t>(comps) == 0 ? '\n' : ' ');
    std::fprintf(f, "</DataArray>\n");
}

}  // namespace

void DataOut::write_vtu(const std::string& fileName) {
    FILE* f = std::fopen(fileName.c_str(), "w");
    if (!f) throw std::runtime_error("cannot write " + fileName);
    const std::size_t nn = opVerticesAll.size(), ne = opTriaHex.size();
    std::fprintf(f, "<?xml version=\"1.0\"?>\n<VTKFile type=\"UnstructuredGrid\" version=\"0.1\" "
                    "byte_order=\"LittleEndian\">\n<UnstructuredGrid>\n");
    std::fprintf(f, "<FieldData>\n<DataArray type=\"Float64\" Name=\"TimeValue\" NumberOfTuples=\"1\" "
                    "format=\"ascii\">%.17g</DataArray>\n</FieldData>\n", time);
    std::fprintf(f, "<Piece NumberOfPoints=\"%zu\" NumberOfCells=\"%zu\">\n", nn, ne);
    std::fprintf(f, "<PointData>\n");
    for (std::size_t i = 0; i < opVec.size(); ++i) write_array(f, opName[i], components(opDataType[i]), opVec[i], nn);
    std::fprintf(f, "</PointData>\n<CellData>\n");
    for (std::size_t i = 0; i < opVec_Ele.size(); ++i)
        write_array(f, opName_Ele[i], components(opDataType_Ele[i]), opVec_Ele[i], ne);
    std::fprintf(f, "</CellData>\n<Points>\n<DataArray type=\"Float64\" NumberOfComponents=\"3\" format=\"ascii\">\n");
    for (const auto& p : opVerticesAll) std::fprintf(f, "%.17g %.17g %.17g\n", p[0], p[1], p[2]);
    std::fprintf(f, "</DataArray>\n</Points>\n<Cells>\n"
                    "<DataArray type=\"Int64\" Name=\"connectivity\" format=\"ascii\">\n");
    for (const auto& el : opTriaHex) {
        const auto& vi = el.get_verticesIndex();
        for (std::size_t k = 0; k < vi.size(); ++k)
            std::fprintf(f, "%u%c", static_cast<unsigned>(vi[k]), k + 1 == vi.size() ? '\n' : ' ');
    }
    std::fprintf(f, "</DataArray>\n<DataArray type=\"Int64\" Name=\"offsets\" format=\"ascii\">\n");
    std::size_t off = 0;
    for (const auto& el : opTriaHex) {
        off += el.get_verticesIndex().size();
        std::fprintf(f, "%zu\n", off);
    }
    std::fprintf(f, "</DataArray>\n<DataArray type=\"UInt8\" Name=\"types\" format=\"ascii\">\n");
    for (std::size_t e = 0; e < ne; ++e) std::fprintf(f, "12\n");
    std::fprintf(f, "</DataArray>\n</Cells>\n</Piece>\n</UnstructuredGrid>\n</VTKFile>\n");
    std::fclose(f);
}

void DataOut::write_vtu_virtualParticles(const unsigned int&, const FSI_share_data&) const {}

}  // namespace EnSC
