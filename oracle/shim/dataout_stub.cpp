// Test infrastructure (oracle build only): a VTK-free stand-in for the
// reference's DataOut class (Explicit3D/include/dataOut.h:44-97).
//
// The reference writes .vtu files through VTK (Explicit3D/source/dataOut.cpp),
// which cannot be linked on Linux.  Output is off the stepper's hot path
// (exDyna3D::output_results only reads state), so the oracle harness links
// this stub instead: it keeps the declared interface and writes nothing.
#include "dataOut.h"

namespace EnSC {

DataOut::DataOut(const Types::VerticesAll<3>& pVerticesAll,
                 const std::vector<Element_HexN8>& pTriaHex, Types::Real t)
    : opVerticesAll(pVerticesAll), opTriaHex(pTriaHex), time(t) {}

void DataOut::add_node_data(DataOutType::DataType dataType,
                            const Eigen::Matrix<Types::Real, Eigen::Dynamic, 1>* vec,
                            std::string name) {
    opDataType.push_back(dataType);
    opVec.push_back(vec);
    opName.push_back(name);
}

void DataOut::add_ele_data(DataOutType::DataType dataType,
                           const Eigen::Matrix<Types::Real, Eigen::Dynamic, 1>* vec,
                           std::string name) {
    opDataType_Ele.push_back(dataType);
    opVec_Ele.push_back(vec);
    opName_Ele.push_back(name);
}

void DataOut::write_vtu(const std::string&) {}

void DataOut::write_vtu_virtualParticles(const unsigned int&, const FSI_share_data&) const {}

}  // namespace EnSC
