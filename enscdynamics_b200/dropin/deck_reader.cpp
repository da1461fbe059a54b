// DataInFast: see deck_reader.h.  Each handler below states the reference
// handler it follows (Explicit3D/source/dataIn.cpp).
#include "deck_reader.h"

#include <algorithm>
#include <cctype>
#include <cerrno>
#include <charconv>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>

namespace EnSC {

namespace {

void upper(std::string& s) {
    for (char& c : s) c = static_cast<char>(std::toupper(static_cast<unsigned char>(c)));
}

void remove_spaces(std::string& s) {
    s.erase(std::remove_if(s.begin(), s.end(), [](unsigned char c) { return std::isspace(c) != 0; }), s.end());
}

bool contains(const std::string& s, const char* key) { return s.find(key) != std::string::npos; }

// extractNameFromKeyword (dataIn.cpp:101-115): the text after `prefix` up to
// the next comma, without white space
std::string name_after(const std::string& line, const std::string& prefix = "NAME=") {
    std::size_t p = line.find(prefix);
    if (p == std::string::npos) return std::string();
    p += prefix.size();
    std::size_t e = line.find(',', p);
    if (e == std::string::npos) e = line.size();
    std::string r = line.substr(p, e - p);
    remove_spaces(r);
    return r;
}

// Comma-separated fields as std::getline(stream, token, ',') yields them:
// a trailing comma (or an empty line) gives no final empty field.
class Fields {
public:
    Fields(const char* b, const char* e) : p_(b), e_(e) {}
    explicit Fields(const std::string& s) : p_(s.data()), e_(s.data() + s.size()) {}
    // next field as [b, e); false when none is left
    bool next(const char*& b, const char*& e) {
        if (p_ >= e_) return false;
        b = p_;
        const char* c = static_cast<const char*>(std::memchr(p_, ',', static_cast<std::size_t>(e_ - p_)));
        if (c) {
            e = c;
            p_ = c + 1;
        } else {
            e = e_;
            p_ = e_;
        }
        return true;
    }
    bool next(std::string& out) {
        const char *b, *e;
        if (!next(b, e)) {
            out.clear();
            return false;
        }
        out.assign(b, e);
        return true;
    }

private:
    const char* p_;
    const char* e_;
};

[[noreturn]] void bad_number(const char* b, const char* e) {
    throw std::runtime_error("deck: not a number: '" + std::string(b, e) + "'");
}

// std::stod on the field [b, e): leading white space, then the longest
// number strtod accepts; no number or a value out of range throws (as stod).
// Decimal numbers go through std::from_chars, which rounds correctly as
// strtod does (same bits), about five times faster; anything else (a '+'
// sign, hexadecimal, a result out of range) through strtod itself.
double to_double(const char* b, const char* e) {
    while (b < e && std::isspace(static_cast<unsigned char>(*b))) ++b;
    if (b == e) bad_number(b, e);
    if (*b != '+') {
        double v;
        const auto r = std::from_chars(b, e, v, std::chars_format::general);
        if (r.ec == std::errc() && !(r.ptr < e && (*r.ptr == 'x' || *r.ptr == 'X'))) return v;
    }
    char tmp[64];
    const char* s = b;
    const std::size_t n = static_cast<std::size_t>(e - b);
    std::string big;
    if (n < sizeof(tmp)) {  // a terminated copy: strtod must not run past the field
        std::memcpy(tmp, b, n);
        tmp[n] = '\0';
        s = tmp;
    } else {
        big.assign(b, e);
        s = big.c_str();
    }
    char* end = nullptr;
    errno = 0;
    const double v = std::strtod(s, &end);
    if (end == s || errno == ERANGE) bad_number(b, e);
    return v;
}
double to_double(const std::string& s) { return to_double(s.data(), s.data() + s.size()); }

// std::stoul / std::stoi on a field
unsigned long to_ulong(const char* b, const char* e) {
    while (b < e && std::isspace(static_cast<unsigned char>(*b))) ++b;
    if (b == e) bad_number(b, e);
    // digits only: the common case
    unsigned long v = 0;
    const char* p = b;
    while (p < e && *p >= '0' && *p <= '9' && v < 100000000000000000ul) v = v * 10 + static_cast<unsigned long>(*p++ - '0');
    if (p > b && (p == e || !(*p >= '0' && *p <= '9'))) return v;
    std::string t(b, e);
    char* end = nullptr;
    errno = 0;
    const unsigned long r = std::strtoul(t.c_str(), &end, 10);
    if (end == t.c_str() || errno == ERANGE) bad_number(b, e);
    return r;
}
int to_int(const std::string& s) {
    // a few plain digits: the common case
    if (!s.empty() && s.size() <= 9) {
        std::size_t i = 0;
        while (i < s.size() && s[i] == ' ') ++i;
        int v = 0;
        std::size_t j = i;
        while (j < s.size() && s[j] >= '0' && s[j] <= '9') v = v * 10 + (s[j++] - '0');
        if (j > i && (j == s.size() || s[j] == ' ')) return v;
    }
    const char* b = s.c_str();
    char* end = nullptr;
    errno = 0;
    const long r = std::strtol(b, &end, 10);
    if (end == b || errno == ERANGE || r < INT32_MIN || r > INT32_MAX) bad_number(s.data(), s.data() + s.size());
    return static_cast<int>(r);
}

// std::stoul that reports failure instead of throwing (the set lists catch)
bool try_ulong(const std::string& t, unsigned long& out) {
    const char* b = t.c_str();
    char* end = nullptr;
    errno = 0;
    const unsigned long r = std::strtoul(b, &end, 10);
    if (end == b || errno == ERANGE) return false;
    out = r;
    return true;
}

// The numbers of a set-list line (dataIn.cpp:684-695): white-space separated
// words, one trailing comma removed, each read as an unsigned prefix; words
// that hold no number are skipped.
void set_line_values(const std::string& line, std::vector<std::size_t>& out) {
    std::size_t i = 0;
    const std::size_t n = line.size();
    std::string w;
    while (i < n) {
        while (i < n && std::isspace(static_cast<unsigned char>(line[i]))) ++i;
        if (i >= n) break;
        std::size_t j = i;
        while (j < n && !std::isspace(static_cast<unsigned char>(line[j]))) ++j;
        w.assign(line, i, j - i);
        if (w.back() == ',') w.pop_back();
        unsigned long v;
        if (try_ulong(w, v)) out.push_back(v);
        i = j;
    }
}

// istream >> double as INSTANCE's translation line reads it
bool read_double(const char*& p, const char* e, double& v) {
    while (p < e && std::isspace(static_cast<unsigned char>(*p))) ++p;
    if (p >= e || !(std::isdigit(static_cast<unsigned char>(*p)) || *p == '+' || *p == '-' || *p == '.')) return false;
    std::string t(p, e);
    char* end = nullptr;
    v = std::strtod(t.c_str(), &end);
    if (end == t.c_str()) return false;
    p += end - t.c_str();
    return true;
}

}  // namespace

DataInFast::DataInFast(exDyna3D_GPU& model) : m_(model) {}

bool DataInFast::getline(std::string& out) {
    if (pos_ >= buf_.size()) {
        out.clear();
        return false;
    }
    const char* b = buf_.data() + pos_;
    const char* nl = static_cast<const char*>(std::memchr(b, '\n', buf_.size() - pos_));
    const std::size_t len = nl ? static_cast<std::size_t>(nl - b) : buf_.size() - pos_;
    out.assign(b, len);
    pos_ += len + (nl ? 1 : 0);
    return true;
}

std::size_t DataInFast::block_lines() const {
    std::size_t n = 0, p = pos_;
    const std::size_t size = buf_.size();
    while (p < size && buf_[p] != '*') {
        ++n;
        const void* nl = std::memchr(buf_.data() + p, '\n', size - p);
        if (!nl) break;
        p = static_cast<std::size_t>(static_cast<const char*>(nl) - buf_.data()) + 1;
    }
    return n;
}

void DataInFast::skip_line() {
    if (pos_ >= buf_.size()) return;
    const char* b = buf_.data() + pos_;
    const char* nl = static_cast<const char*>(std::memchr(b, '\n', buf_.size() - pos_));
    pos_ = nl ? static_cast<std::size_t>(nl - buf_.data()) + 1 : buf_.size();
}

// read_inp (dataIn.cpp:300-558)
void DataInFast::read_inp(const std::string& fileName) {
    FILE* f = std::fopen(fileName.c_str(), "rb");
    if (!f) throw std::runtime_error("cannot open deck " + fileName);
    std::fseek(f, 0, SEEK_END);
    const long size = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    buf_.resize(size > 0 ? static_cast<std::size_t>(size) : 0);
    const std::size_t got = buf_.empty() ? 0 : std::fread(&buf_[0], 1, buf_.size(), f);
    std::fclose(f);
    if (got != buf_.size()) throw std::runtime_error("cannot read deck " + fileName);
    pos_ = 0;
    state_ = State::GLOBAL;
    parts_.clear();
    assemblies_.clear();
    part_ = nullptr;
    assembly_ = nullptr;

    StepData initial;
    initial.name = "Initial";
    initial.timePeriod = 0.0;
    m_.steps.push_back(initial);

    while (!at_end()) {
        if (peek() == '*') {
            getline(str_);
            if (str_.size() > 1 && str_[1] != '*') {
                upper(str_);
                dispatch();
            }
        } else {
            skip_line();
        }
    }
    transfer();
    m_.mMatElastic.update();
}

void DataInFast::dispatch() {
    // the structure keywords first, in the reference's order
    if (contains(str_, "*HEADING")) {
        while (peek() != '*' && !at_end()) skip_line();
        return;
    }
    if (contains(str_, "*PART")) {
        parts_.emplace_back();
        parts_.back().name = name_after(str_);
        part_ = &parts_.back();
        state_ = State::PART;
        return;
    }
    if (contains(str_, "*ASSEMBLY")) {
        std::string name = name_after(str_);
        if (name.empty()) name = "MainAssembly";
        assemblies_.emplace_back();
        assemblies_.back().name = name;
        assembly_ = &assemblies_.back();
        state_ = State::ASSEMBLY;
        return;
    }
    if (contains(str_, "*MATERIAL")) {
        state_ = State::MATERIAL;
        return;
    }
    if (contains(str_, "*STEP")) {
        std::string name = name_after(str_);
        if (name.empty()) name = "Step-" + std::to_string(m_.steps.size() + 1);
        state_ = State::STEP;
        StepData sd;
        sd.name = name;
        m_.steps.push_back(sd);
        return;
    }
    if (contains(str_, "*INITIAL CONDITIONS")) state_ = State::PREDEFINED;

    // the keyword table, in its (alphabetical) order: the first keyword the
    // line contains picks the handler (dataIn.cpp:392-401)
    if (contains(str_, "*AMPLITUDE")) return amplitude();
    if (contains(str_, "*BOUNDARY")) return boundary();
    if (contains(str_, "*BULK VISCOSITY")) return bulk_viscosity();
    if (contains(str_, "*DLOAD")) return dload();
    if (contains(str_, "*DSLOAD")) return dsload();
    if (contains(str_, "*DYNAMIC")) return dynamic();
    if (contains(str_, "*ELEMENT")) return element_block();
    if (contains(str_, "*ELSET")) return element_set();
    if (contains(str_, "*END ASSEMBLY")) {
        assembly_ = nullptr;
        state_ = State::GLOBAL;
        return;
    }
    if (contains(str_, "*END INSTANCE")) return;
    if (contains(str_, "*END PART")) {
        part_ = nullptr;
        state_ = State::GLOBAL;
        return;
    }
    if (contains(str_, "*END STEP")) {
        state_ = State::GLOBAL;
        return;
    }
    if (contains(str_, "*INITIAL CONDITION")) {
        // INITIAL_CONDITIONS (:790-798)
        if (contains(str_, "TYPE") && contains(str_, "VELOCITY")) initial_velocity();
        return;
    }
    if (contains(str_, "*INSTANCE")) return instance();
    if (contains(str_, "*MATERIAL")) return;  // not reached: caught above
    if (contains(str_, "*NODE")) return node_block();
    if (contains(str_, "*NSET")) return node_set();
    if (contains(str_, "*OUTPUT")) return output();  // also takes "*OUTPUT INTERVAL" lines, as the reference
    if (contains(str_, "*SURFACE")) return surface();

    // keywords outside the table, by context (:410-531)
    switch (state_) {
        case State::PART:
            if (contains(str_, "*SOLID SECTION") && peek() != '*' && !at_end()) skip_line();
            break;
        case State::MATERIAL:
            if (contains(str_, "*DENSITY")) {
                if (peek() != '*' && !at_end()) {
                    std::string line;
                    getline(line);
                    const char* p = line.data();
                    double rho = 0.0;
                    if (!read_double(p, line.data() + line.size(), rho)) rho = 0.0;
                    m_.mMatElastic.rho = rho;
                }
            } else if (contains(str_, "*ELASTIC")) {
                if (peek() != '*' && !at_end()) {
                    std::string line, t;
                    getline(line);
                    Fields fl(line);
                    fl.next(t);
                    const double E = to_double(t);
                    fl.next(t);
                    const double nu = to_double(t);
                    m_.mMatElastic.E = E;
                    m_.mMatElastic.v = nu;
                    m_.mMatElastic.update();
                }
            }
            break;
        case State::STEP:
            if (contains(str_, "*RESTART"))
                while (peek() != '*' && !at_end()) skip_line();
            break;
        default:
            break;
    }
}

// NODE (:567-584)
void DataInFast::node_block() {
    if (!part_) return;
    while (peek() == '*') skip_line();
    Part& p = *part_;
    p.nodes.reserve(p.nodes.size() + block_lines());
    while (peek() != '*' && !at_end()) {
        const char* b = line_begin();
        const char* nl = static_cast<const char*>(std::memchr(b, '\n', buf_.size() - pos_));
        const char* e = nl ? nl : buf_.data() + buf_.size();
        pos_ = static_cast<std::size_t>(e - buf_.data()) + (nl ? 1 : 0);
        if (e == b) continue;
        Fields fl(b, e);
        const char *fb, *fe;
        fl.next(fb, fe);  // node number
        std::array<double, 3> x;
        for (int c = 0; c < 3; ++c) {
            if (!fl.next(fb, fe)) bad_number(b, e);
            x[c] = to_double(fb, fe);
        }
        p.nodes.push_back(x);
    }
}

// ELEMENT (:652-669)
void DataInFast::element_block() {
    if (!part_) return;
    while (peek() == '*') skip_line();
    Part& p = *part_;
    if (p.conn_start.empty()) p.conn_start.push_back(0);
    const std::size_t lines = block_lines();
    p.conn_start.reserve(p.conn_start.size() + lines);
    p.conn.reserve(p.conn.size() + 8 * lines);
    while (peek() != '*' && !at_end()) {
        const char* b = line_begin();
        const char* nl = static_cast<const char*>(std::memchr(b, '\n', buf_.size() - pos_));
        const char* e = nl ? nl : buf_.data() + buf_.size();
        pos_ = static_cast<std::size_t>(e - buf_.data()) + (nl ? 1 : 0);
        if (e == b) continue;
        Fields fl(b, e);
        const char *fb, *fe;
        fl.next(fb, fe);  // element number
        while (fl.next(fb, fe)) p.conn.push_back(static_cast<uint32_t>(to_ulong(fb, fe) - 1));
        p.conn_start.push_back(static_cast<uint32_t>(p.conn.size()));
    }
}

// SET_NODE_LIST (:679-726)
void DataInFast::node_set() {
    std::string set = name_after(str_, "NSET=");
    if (set.empty()) set = name_after(str_, "ELSET=");
    const std::string inst = name_after(str_, "INSTANCE=");
    const bool generate = contains(str_, "GENERATE");
    std::vector<std::size_t> nodes;
    std::string line;
    while (peek() != '*' && !at_end()) {
        getline(line);
        if (line.empty()) continue;
        set_line_values(line, nodes);
    }
    if (generate && nodes.size() >= 2) {
        const std::size_t start = nodes[0], end = nodes[1], step = nodes.size() >= 3 ? nodes[2] : 1;
        if (step == 0) throw std::runtime_error("deck: *Nset generate with increment 0");
        nodes.clear();
        for (std::size_t i = start; i <= end; i += step) nodes.push_back(i);
    }
    for (auto& i : nodes) i -= 1;
    if (part_ && state_ == State::PART) return;  // part sets are not carried into the model
    if (assembly_ && state_ == State::ASSEMBLY) {
        if (!inst.empty()) {
            assembly_->node_sets[set][inst] = nodes;
        } else {
            std::map<std::string, std::vector<std::size_t>> g;
            g["__GLOBAL__"] = nodes;
            assembly_->node_sets[set] = g;
        }
    }
}

// SET_ELE_LIST (:1281-1325)
void DataInFast::element_set() {
    std::string set = name_after(str_, "NSET=");
    if (set.empty()) set = name_after(str_, "ELSET=");
    const std::string inst = name_after(str_, "INSTANCE=");
    std::vector<std::size_t> elems, vals;
    std::string line;
    while (peek() != '*' && !at_end()) {
        getline(line);
        if (line.empty()) continue;
        vals.clear();
        set_line_values(line, vals);
        if (vals.size() == 3) {
            if (vals[2] == 0) throw std::runtime_error("deck: *Elset range with increment 0");
            for (std::size_t i = vals[0]; i <= vals[1]; i += vals[2]) elems.push_back(i);
        } else {
            elems.insert(elems.end(), vals.begin(), vals.end());
        }
    }
    for (auto& i : elems) i -= 1;
    if (part_ && state_ == State::PART) return;
    if (assembly_ && state_ == State::ASSEMBLY) {
        if (!inst.empty()) {
            assembly_->element_sets[set][inst] = elems;
        } else {
            std::map<std::string, std::vector<std::size_t>> g;
            g["__GLOBAL__"] = elems;
            assembly_->element_sets[set] = g;
        }
    }
}

// BOUNDARY (:728-781)
void DataInFast::boundary() {
    const bool op_new = contains(str_, "OP=NEW");
    const bool velocity = contains(str_, "TYPE=VELOCITY");
    if (op_new && !m_.steps.empty()) {
        StepData& sd = (state_ == State::STEP) ? m_.steps.back() : m_.steps.front();
        if (velocity) sd.resetVelBoundary = true;
        else sd.resetSpcBoundary = true;
    }
    // a command without data: the next line is empty, a keyword or the end
    const bool empty_cmd = at_end() || peek() == '\n' || peek() == '*';
    if (empty_cmd) return;
    if (velocity) velocity_lines();
    else spc_lines();
}

// SPC_NODE (:902-1022)
void DataInFast::spc_lines() {
    while (peek() == '*') skip_line();
    if (peek() == '*') return;
    std::string line, t;
    while (peek() != '*' && !at_end()) {
        getline(line);
        upper(line);
        std::pair<std::string, std::array<std::size_t, 3>> bc;
        Fields fl(line);
        fl.next(t);
        bc.first = contains(line, "SET-") ? t : "#" + t;
        if (contains(line, "PINNED") || contains(line, "ENCASTRE")) {
            bc.second = {0, 2, 1};
        } else if (contains(line, "XSYMM")) {
            bc.second = {0, 0, 1};
        } else if (contains(line, "YSYMM")) {
            bc.second = {1, 1, 1};
        } else if (contains(line, "ZSYMM")) {
            bc.second = {2, 2, 1};
        } else {
            fl.next(t);
            if (t.empty()) {
                bc.second = {0, 2, 1};
            } else {
                bc.second[0] = static_cast<std::size_t>(to_int(t) - 1);
                fl.next(t);
                bc.second[1] = t.empty() ? bc.second[0] : static_cast<std::size_t>(to_int(t) - 1);
                fl.next(t);
                bc.second[2] = t.empty() ? 1 : static_cast<std::size_t>(to_int(t));
            }
        }
        if (state_ == State::STEP && !m_.steps.empty()) m_.steps.back().boundary.spc_nodes.push_back(bc);
        else if (!m_.steps.empty()) m_.steps.front().boundary.spc_nodes.push_back(bc);
    }
}

// VELOCITY_NODE (:1114-1201)
void DataInFast::velocity_lines() {
    while (peek() == '*') skip_line();
    if (peek() == '*') return;
    std::string line, t;
    while (peek() != '*' && !at_end()) {
        getline(line);
        upper(line);
        std::pair<std::string, std::pair<std::array<std::size_t, 2>, Types::Real>> bc;
        bc.second.first = {0, 0};
        bc.second.second = 0.0;
        Fields fl(line);
        fl.next(t);
        bc.first = contains(line, "SET-") ? t : "#" + t;
        fl.next(t);
        if (t.empty()) continue;  // no DOF given: the line is skipped
        bc.second.first[0] = static_cast<std::size_t>(to_int(t) - 1);
        fl.next(t);
        bc.second.first[1] = t.empty() ? bc.second.first[0] : static_cast<std::size_t>(to_int(t) - 1);
        if (fl.next(t)) bc.second.second = to_double(t);
        if (state_ == State::STEP && !m_.steps.empty()) m_.steps.back().boundary.vel_nodes.push_back(bc);
        else if (!m_.steps.empty()) m_.steps.front().boundary.vel_nodes.push_back(bc);
    }
}

// INITIAL_VELOCITY (:1030-1106)
void DataInFast::initial_velocity() {
    while (peek() == '*') skip_line();
    auto& list = m_.ini_vel_generation;
    list.reserve(list.size() + block_lines());
    std::string ref, dof;
    while (peek() != '*' && !at_end()) {
        const char* b = line_begin();
        const char* nl = static_cast<const char*>(std::memchr(b, '\n', buf_.size() - pos_));
        const char* e = nl ? nl : buf_.data() + buf_.size();
        pos_ = static_cast<std::size_t>(e - buf_.data()) + (nl ? 1 : 0);
        if (e == b) continue;
        Fields fl(b, e);
        const char* fb = nullptr;
        const char* fe = nullptr;
        fl.next(fb, fe);
        // the node or set reference, upper case, without white space (the
        // numeric fields read the same in either case)
        ref.assign(1, '#');
        for (const char* c = fb; c < fe; ++c)
            if (!std::isspace(static_cast<unsigned char>(*c)))
                ref.push_back(static_cast<char>(std::toupper(static_cast<unsigned char>(*c))));
        std::pair<std::string, std::pair<std::size_t, Types::Real>> iv;
        const bool is_set = ref.find("SET-", 1) != std::string::npos;  // also finds "NSET-"
        const std::size_t dot = ref.find('.', 1);
        if (is_set) {
            // "instance.set" stays as written; a set without instance keeps its name
            iv.first = ref.substr(1);
        } else if (dot != std::string::npos) {
            iv.first = "#" + ref.substr(dot + 1);  // a node number after an instance prefix
        } else {
            iv.first = std::move(ref);
        }
        try {
            if (fl.next(fb, fe)) {
                dof.assign(fb, fe);
                iv.second.first = static_cast<std::size_t>(to_int(dof) - 1);
            } else {
                iv.second.first = 0;
            }
            iv.second.second = fl.next(fb, fe) ? to_double(fb, fe) : 0.0;
        } catch (const std::exception&) {
            continue;  // the reference drops a line whose numbers do not read
        }
        list.push_back(std::move(iv));
    }
}

// DLOAD (:808-836) and GRAV (:1203-1233)
void DataInFast::dload() {
    if (contains(str_, "OP=NEW") && state_ == State::STEP && !m_.steps.empty()) m_.steps.back().resetDload = true;
    const std::string amp = name_after(str_, "AMPLITUDE=");
    std::string line, t;
    while (peek() != '*' && !at_end()) {
        getline(line);
        if (!contains(line, "GRAV")) continue;
        Fields fl(line);
        fl.next(t);
        fl.next(t);
        fl.next(t);
        const double value = to_double(t);
        double dir[3];
        for (int c = 0; c < 3; ++c) {
            fl.next(t);
            dir[c] = to_double(t);
        }
        if (state_ == State::STEP && !m_.steps.empty()) {
            auto& g = m_.steps.back().gravity;
            std::get<0>(g) = true;
            std::get<1>(g) = amp;
            std::get<2>(g) = value;
            std::get<3>(g) = dir[0];
            std::get<4>(g) = dir[1];
            std::get<5>(g) = dir[2];
        }
    }
}

// DSLOAD (:1425-1478)
void DataInFast::dsload() {
    if (contains(str_, "OP=NEW") && state_ == State::STEP && !m_.steps.empty()) m_.steps.back().resetDsload = true;
    const std::string amp = name_after(str_, "AMPLITUDE=");
    std::string line, surf, type, t;
    while (peek() != '*' && !at_end()) {
        getline(line);
        upper(line);
        Fields fl(line);
        fl.next(surf);
        remove_spaces(surf);
        fl.next(type);
        remove_spaces(type);
        fl.next(t);
        const double value = to_double(t);
        if (state_ == State::STEP && !m_.steps.empty()) m_.steps.back().dsload.emplace_back(surf, type, amp, value);
    }
}

// TIME (:844-872)
void DataInFast::dynamic() {
    while (peek() == '*') skip_line();
    std::string line, t;
    while (peek() != '*' && !at_end()) {
        getline(line);
        Fields fl(line);
        fl.next(t);
        fl.next(t);
        const double period = to_double(t);
        if (state_ == State::STEP && !m_.steps.empty()) m_.steps.back().timePeriod = period;
        m_.totalTime += period;
    }
}

// AMP (:1242-1270): each data line replaces the curve
void DataInFast::amplitude() {
    const std::string name = name_after(str_);
    std::string line, t;
    while (peek() != '*' && !at_end()) {
        getline(line);
        int n = 0;
        {
            Fields c(line);
            while (c.next(t)) ++n;
        }
        std::vector<std::array<Types::Real, 2>> pts(static_cast<std::size_t>(n / 2));
        Fields fl(line);
        for (auto& pt : pts) {
            fl.next(t);
            pt[0] = to_double(t);
            fl.next(t);
            pt[1] = to_double(t);
        }
        m_.map_amp_list[name] = pts;
    }
}

// SURFACE (:1339-1417)
void DataInFast::surface() {
    std::string name = name_after(str_, "NAME=");
    const std::string inst = name_after(str_, "INSTANCE=");
    const std::string type_all = name_after(str_, "TYPE=");
    if (name.empty()) {
        while (peek() != '*' && !at_end()) skip_line();
        return;
    }
    remove_spaces(name);
    const std::string full = inst.empty() ? name : inst + "." + name;
    std::string line, set, face;
    while (peek() != '*' && !at_end()) {
        getline(line);
        if (line.empty()) continue;
        upper(line);
        Fields fl(line);
        fl.next(set);
        remove_spaces(set);
        std::string set_inst = inst;
        const std::size_t dot = set.find('.');
        if (dot != std::string::npos) {
            set_inst = set.substr(0, dot);
            set = set.substr(dot + 1);
        }
        fl.next(face);
        remove_spaces(face);
        if (face.empty() && !type_all.empty()) face = type_all;
        const std::string full_set = set_inst.empty() ? set : set_inst + "." + set;
        m_.map_set_surface_list[full] = std::make_pair(full_set, face);
    }
}

// BULK_VISCOSITY (:881-895): the line after the keyword
void DataInFast::bulk_viscosity() {
    std::string line, t;
    getline(line);
    Fields fl(line);
    fl.next(t);
    m_.Cvisl = to_double(t);
    fl.next(t);
    m_.Cvisq = to_double(t);
}

// OUTPUT (:1506-1548)
void DataInFast::output() {
    const std::size_t p = str_.find("NUMBER INTERVAL=");
    if (p != std::string::npos) {
        std::string s = str_.substr(p + 16);
        const std::size_t e = s.find_first_of(", ");
        if (e != std::string::npos) s = s.substr(0, e);
        try {
            const int n = to_int(s);
            if (n > 0) {
                m_.time_interval = m_.totalTime / n;
                m_.time_interval_set = true;
            }
        } catch (const std::exception&) {
        }
    }
    while (peek() != '*' && !at_end()) skip_line();
}

// INSTANCE (:145-205): an optional translation line of three numbers
void DataInFast::instance() {
    if (!assembly_) return;
    Instance in;
    in.name = name_after(str_, "NAME=");
    in.part = name_after(str_, "PART=");
    if (peek() != '*' && !at_end()) {
        const std::size_t here = pos_;
        std::string line;
        getline(line);
        const char* p = line.data();
        const char* e = line.data() + line.size();
        double x, y, z;
        bool ok = read_double(p, e, x);
        if (ok && p < e && *p == ',') ++p;
        ok = ok && read_double(p, e, y);
        if (ok && p < e && *p == ',') ++p;
        ok = ok && read_double(p, e, z);
        if (ok) in.translation = {x, y, z};
        else pos_ = here;
    }
    assembly_->instances.push_back(in);
}

// transferToExDyna (:1550-1790)
void DataInFast::transfer() {
    if (parts_.empty()) return;
    std::size_t total_nodes = 0, total_elems = 0;
    for (const Part& p : parts_) {
        total_nodes += p.nodes.size();
        total_elems += p.conn_start.empty() ? 0 : p.conn_start.size() - 1;
    }
    m_.vertices.clear();
    m_.hexahedron_elements.clear();
    m_.vertices.reserve(total_nodes);
    m_.hexahedron_elements.reserve(total_elems);
    std::vector<Types::Vertex_index> idx;
    auto add_elements = [&](const Part& p, std::size_t offset) {
        const std::size_t n = p.conn_start.empty() ? 0 : p.conn_start.size() - 1;
        for (std::size_t e = 0; e < n; ++e) {
            m_.hexahedron_elements.emplace_back();
            Element_HexN8& el = m_.hexahedron_elements.back();
            el.set_PID(1);
            el.set_MID(1);
            idx.assign(p.conn.begin() + p.conn_start[e], p.conn.begin() + p.conn_start[e + 1]);
            for (auto& v : idx) v = static_cast<Types::Vertex_index>(v + offset);
            el.set_verticesIndex(idx);
        }
    };
    if (!assemblies_.empty()) {
        for (Assembly& a : assemblies_) {
            std::size_t g_node = 0, g_elem = 0;
            for (Instance& in : a.instances) {
                auto it = std::find_if(parts_.begin(), parts_.end(), [&](const Part& p) { return p.name == in.part; });
                if (it == parts_.end()) continue;
                in.node_start = g_node;
                in.element_start = g_elem;
                const bool shift = in.translation[0] != 0.0 || in.translation[1] != 0.0 || in.translation[2] != 0.0;
                for (const auto& x : it->nodes) {
                    Types::Point<3> y = x;
                    if (shift) {
                        y[0] += in.translation[0];
                        y[1] += in.translation[1];
                        y[2] += in.translation[2];
                    }
                    m_.vertices.push_back(y);
                    ++g_node;
                }
                add_elements(*it, in.node_start);
                g_elem += it->conn_start.empty() ? 0 : it->conn_start.size() - 1;
            }
            auto global_sets = [&](const std::map<std::string, std::map<std::string, std::vector<std::size_t>>>& sets,
                                   bool nodes, std::map<std::string, std::vector<std::size_t>>& out) {
                for (const auto& s : sets) {
                    std::vector<std::size_t> all;
                    for (const auto& part : s.second) {
                        if (part.first == "__GLOBAL__") {
                            all.insert(all.end(), part.second.begin(), part.second.end());
                            continue;
                        }
                        auto in = std::find_if(a.instances.begin(), a.instances.end(),
                                               [&](const Instance& i) { return i.name == part.first; });
                        if (in == a.instances.end()) continue;
                        const std::size_t off = nodes ? in->node_start : in->element_start;
                        for (std::size_t v : part.second) all.push_back(v + off);
                    }
                    out[s.first] = all;
                }
            };
            global_sets(a.node_sets, true, m_.map_set_node_list);
            global_sets(a.element_sets, false, m_.map_set_ele_list);
        }
    } else {
        std::map<std::string, std::size_t> node_off;
        std::size_t g_node = 0;
        for (const Part& p : parts_) {
            node_off[p.name] = g_node;
            for (const auto& x : p.nodes) {
                m_.vertices.push_back(x);
                ++g_node;
            }
        }
        for (const Part& p : parts_) add_elements(p, node_off[p.name]);
    }
}

}  // namespace EnSC
