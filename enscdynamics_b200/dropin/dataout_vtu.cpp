// DataOut without VTK: the reference's result writer interface
// (Explicit3D/include/dataOut.h:44-97) writing VTK XML unstructured-grid files
// (.vtu, inline base64 "binary" arrays with UInt64 headers) directly.  The reference builds these files through the VTK
// library (Explicit3D/source/dataOut.cpp), which the GPU drop-in does not
// link; the written file carries the same mesh, node fields and element
// fields: points, hexahedra (VTK cell type 12) with the reference's local node
// order, which is VTK's, one PointData array per add_node_data call and one
// CellData array per add_ele_data call (scalar: 1 component, vector: 3,
// symmetric tensor: 6), and the time as FieldData "TimeValue".
// write_vtu_virtualParticles writes nothing: there are no FSI particles.
#include "dataOut.h"

#include <cstdint>
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

// VTK XML "binary" data: base64 of a UInt64 byte count followed by the raw
// little-endian values, inline in the DataArray element.
class Base64Out {
public:
    explicit Base64Out(FILE* f) : f_(f) {}
    void bytes(const void* p, std::size_t n) {
        const unsigned char* b = static_cast<const unsigned char*>(p);
        for (std::size_t i = 0; i < n; ++i) {
            acc_[na_++] = b[i];
            if (na_ == 3) emit(3);
        }
    }
    void finish() {
        if (na_ > 0) emit(na_);
        if (nbuf_) std::fwrite(buf_, 1, nbuf_, f_);
        nbuf_ = 0;
    }

private:
    // one group of up to 3 bytes as 4 characters ('=' padding)
    void emit(int n) {
        static const char* kAlpha = "ABCDEFGHIJKLMNOPQRSTUVWXYZabcdefghijklmnopqrstuvwxyz0123456789+/";
        const unsigned v = (acc_[0] << 16) | ((n > 1 ? acc_[1] : 0u) << 8) | (n > 2 ? acc_[2] : 0u);
        if (nbuf_ + 4 > sizeof(buf_)) {
            std::fwrite(buf_, 1, nbuf_, f_);
            nbuf_ = 0;
        }
        buf_[nbuf_++] = kAlpha[(v >> 18) & 63];
        buf_[nbuf_++] = kAlpha[(v >> 12) & 63];
        buf_[nbuf_++] = n > 1 ? kAlpha[(v >> 6) & 63] : '=';
        buf_[nbuf_++] = n > 2 ? kAlpha[v & 63] : '=';
        na_ = 0;
    }
    FILE* f_;
    unsigned acc_[3] = {0, 0, 0};
    int na_ = 0;
    char buf_[1 << 16];
    std::size_t nbuf_ = 0;
};

// One DataArray of `count` values of type T, value i given by get(i).
template <typename T, typename Get>
void write_binary_array(FILE* f, const char* type, const std::string& name, int comps, std::size_t count, Get get) {
    if (name.empty())
        std::fprintf(f, "<DataArray type=\"%s\" NumberOfComponents=\"%d\" format=\"binary\">\n", type, comps);
    else
        std::fprintf(f, "<DataArray type=\"%s\" Name=\"%s\" NumberOfComponents=\"%d\" format=\"binary\">\n", type,
                     name.c_str(), comps);
    Base64Out b(f);
    const uint64_t nbytes = static_cast<uint64_t>(count) * sizeof(T);
    b.bytes(&nbytes, sizeof nbytes);
    T chunk[1024];
    std::size_t k = 0;
    for (std::size_t i = 0; i < count; ++i) {
        chunk[k++] = get(i);
        if (k == 1024) {
            b.bytes(chunk, sizeof chunk);
            k = 0;
        }
    }
    b.bytes(chunk, k * sizeof(T));
    b.finish();
    std::fprintf(f, "\n</DataArray>\n");
}

void write_field(FILE* f, const std::string& name, int comps, const Eigen::Matrix<Types::Real, Eigen::Dynamic, 1>* v,
                 std::size_t n_items) {
    const std::size_t have = v ? static_cast<std::size_t>(v->size()) : 0;
    write_binary_array<double>(f, "Float64", name, comps, n_items * static_cast<std::size_t>(comps),
                               [&](std::size_t i) { return i < have ? (*v)[static_cast<Eigen::Index>(i)] : 0.0; });
}

}  // namespace

void DataOut::write_vtu(const std::string& fileName) {
    FILE* f = std::fopen(fileName.c_str(), "wb");
    if (!f) throw std::runtime_error("cannot write " + fileName);
    const std::size_t nn = opVerticesAll.size(), ne = opTriaHex.size();
    std::fprintf(f, "<?xml version=\"1.0\"?>\n<VTKFile type=\"UnstructuredGrid\" version=\"1.0\" "
                    "byte_order=\"LittleEndian\" header_type=\"UInt64\">\n<UnstructuredGrid>\n");
    std::fprintf(f, "<FieldData>\n<DataArray type=\"Float64\" Name=\"TimeValue\" NumberOfTuples=\"1\" "
                    "format=\"ascii\">%.17g</DataArray>\n</FieldData>\n", time);
    std::fprintf(f, "<Piece NumberOfPoints=\"%zu\" NumberOfCells=\"%zu\">\n", nn, ne);
    std::fprintf(f, "<PointData>\n");
    for (std::size_t i = 0; i < opVec.size(); ++i) write_field(f, opName[i], components(opDataType[i]), opVec[i], nn);
    std::fprintf(f, "</PointData>\n<CellData>\n");
    for (std::size_t i = 0; i < opVec_Ele.size(); ++i)
        write_field(f, opName_Ele[i], components(opDataType_Ele[i]), opVec_Ele[i], ne);
    std::fprintf(f, "</CellData>\n<Points>\n");
    write_binary_array<double>(f, "Float64", "", 3, 3 * nn,
                               [&](std::size_t i) { return opVerticesAll[i / 3][static_cast<int>(i % 3)]; });
    std::fprintf(f, "</Points>\n<Cells>\n");
    write_binary_array<int64_t>(f, "Int64", "connectivity", 1, 8 * ne, [&](std::size_t i) {
        return static_cast<int64_t>(opTriaHex[i / 8].get_verticesIndex()[i % 8]);
    });
    write_binary_array<int64_t>(f, "Int64", "offsets", 1, ne,
                                [&](std::size_t i) { return static_cast<int64_t>(8 * (i + 1)); });
    write_binary_array<uint8_t>(f, "UInt8", "types", 1, ne, [](std::size_t) { return static_cast<uint8_t>(12); });
    std::fprintf(f, "</Cells>\n</Piece>\n</UnstructuredGrid>\n</VTKFile>\n");
    std::fclose(f);
}

void DataOut::write_vtu_virtualParticles(const unsigned int&, const FSI_share_data&) const {}

}  // namespace EnSC
