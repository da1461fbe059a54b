// DataInFast: the reference's deck reader interface (Explicit3D/include/
// dataIn.h:35-41: constructed on a solver, read_inp(fileName)) with a faster
// implementation, for the GPU drop-in.
//
// The reference reader (Explicit3D/source/dataIn.cpp:300-558) reads a deck
// line by line through std::ifstream, builds an std::istringstream per data
// line and keeps every part's nodes and elements in intermediate structures
// before copying them into the solver.  On a 500k-element deck that takes
// longer than the GPU needs for thousands of cycles, so it sets the time to
// the first cycle.  This reader loads the file once, walks its lines in
// memory and converts numbers in place (strtod / strtoul, the conversions
// behind the reference's std::stod / std::stoul, so values are the same bit
// for bit), and fills the same solver members with the same values in the
// same order: nodes, hexahedra, assembly node and element sets, surfaces,
// steps (period, displacement and velocity conditions, reset flags, gravity,
// distributed surface loads), initial velocities, amplitudes, material,
// bulk viscosity, total time and output interval.
//
// It follows the reference's parsing rules, including the ones that are
// easy to miss: keyword lines are upper-cased and dispatched to the first
// handler (in the reference's alphabetical table) whose keyword they contain;
// handlers that skip '*' lines before their data also skip a keyword line
// there; part-level sets are not carried into the solver; an amplitude keeps
// only its last data line; a data line of a set list contributes only the
// numbers that whitespace separates.  ensc_reader_bench checks a deck by
// reading it with both readers and comparing every member they fill.
//
// Malformed numeric fields that make the reference throw (and terminate)
// raise std::runtime_error here.
#pragma once

#include "exDyna3D_GPU.h"

#include <array>
#include <cstdint>
#include <map>
#include <string>
#include <vector>

namespace EnSC {

class DataInFast {
public:
    explicit DataInFast(exDyna3D_GPU& model);
    void read_inp(const std::string& fileName);

private:
    enum class State { GLOBAL, PART, ASSEMBLY, STEP, MATERIAL, PREDEFINED };
    struct Part {
        std::string name;
        std::vector<std::array<double, 3>> nodes;
        std::vector<uint32_t> conn;          // element node indices, 0-based, concatenated
        std::vector<uint32_t> conn_start;    // element e's nodes: conn[conn_start[e] .. conn_start[e + 1])
    };
    struct Instance {
        std::string name, part;
        std::array<double, 3> translation{{0.0, 0.0, 0.0}};
        std::size_t node_start = 0, element_start = 0;
    };
    struct Assembly {
        std::string name;
        std::vector<Instance> instances;
        std::map<std::string, std::map<std::string, std::vector<std::size_t>>> node_sets, element_sets;
    };

    // line cursor over the file
    int peek() const { return pos_ < buf_.size() ? static_cast<unsigned char>(buf_[pos_]) : -1; }
    bool at_end() const { return pos_ >= buf_.size(); }
    bool getline(std::string& out);
    void skip_line();
    // span of the next line without consuming it
    const char* line_begin() const { return buf_.data() + pos_; }
    // lines from the cursor up to the next line that starts with '*' (for
    // reserving the arrays a data block fills)
    std::size_t block_lines() const;

    void dispatch();
    void node_block();
    void element_block();
    void node_set();
    void element_set();
    void boundary();
    void spc_lines();
    void velocity_lines();
    void initial_velocity();
    void dload();
    void dsload();
    void dynamic();
    void amplitude();
    void surface();
    void bulk_viscosity();
    void output();
    void instance();
    void transfer();

    exDyna3D_GPU& m_;
    std::string buf_;
    std::size_t pos_ = 0;
    std::string str_;                        // the current keyword line (upper case)
    State state_ = State::GLOBAL;
    std::vector<Part> parts_;
    std::vector<Assembly> assemblies_;
    Part* part_ = nullptr;
    Assembly* assembly_ = nullptr;
};

}  // namespace EnSC
