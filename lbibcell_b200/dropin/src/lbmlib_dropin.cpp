// libLbmLib — LBIBCell's application API (SimulationRunner, GeometryHandler,
// Geometry, ForceSolver, the plugin registries, the VTK reporters and the
// global parameters) over the lbibcell_b200 device runtime.  Applications
// written against the reference (apps/tutorial_01.cpp) compile against the
// headers in lbibcell_b200/dropin/include and link this library; the time
// loop runs on the GPU through the C ABI of include/lbibcell.h, and bio
// solver plugins that the device does not provide run on the host between
// steps.
#include <LbmLib/include/GlobalSimulationParameters.hpp>
#include <LbmLib/include/SimulationRunner.hpp>
#include <LbmLib/include/geometry/Geometry.hpp>
#include <LbmLib/include/geometry/GeometryHandler.hpp>
#include <LbmLib/include/reportHandler/ReportHandler.hpp>
#include <LbmLib/include/reportHandler/vtkReporterBlock.hpp>
#include <LbmLib/include/solver/BioSolver/BioSolverFactory.hpp>
#include <LbmLib/include/solver/ForceSolver.hpp>
#include <UtilLib/include/Exception.hpp>
#include <UtilLib/include/Log.hpp>

#include <lbibcell.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <ctime>
#include <fstream>
#include <iomanip>
#include <iostream>
#include <set>
#include <sstream>
#include <unistd.h>

// ---------------------------------------------------------------------------
// UtilLib::Log

namespace UtilLib {
namespace {
std::shared_ptr<std::ostream>& logStream() {
    static std::shared_ptr<std::ostream> s;
    return s;
}
LogLevel& logLevel() {
    static LogLevel l = logDEBUG1;
    return l;
}
const char* levelName(LogLevel l) {
    static const char* names[] = {"ERROR", "WARNING", "INFO", "DEBUG", "DEBUG1", "DEBUG2", "DEBUG3", "DEBUG4"};
    return names[(int)l];
}
}  // namespace

Log::~Log() { writeOutput(buffer_.str()); }

std::ostringstream& Log::writeReport(LogLevel level) {
    const std::time_t now = std::time(nullptr);
    char stamp[64];
    std::strftime(stamp, sizeof stamp, "%x %H:%M:%S", std::localtime(&now));
    buffer_ << "- " << stamp << " " << levelName(level) << ":\t";
    return buffer_;
}

std::shared_ptr<std::ostream> Log::getStream() { return logStream(); }
void Log::setStream(std::shared_ptr<std::ostream> pStream) { logStream() = pStream; }
LogLevel Log::getReportingLevel() { return logLevel(); }
void Log::setReportingLevel(LogLevel level) { logLevel() = level; }
void Log::writeOutput(const std::string& msg) {
    if (logStream()) (*logStream()) << msg << std::endl;
}
}  // namespace UtilLib

namespace LbmLib {
namespace {

// Throws the reference's exception with the device runtime's message.
void check(lbib_handle* h, int rc, const char* what) {
    if (rc == LBIB_OK) return;
    char buf[512] = {0};
    long long index = -1;
    if (h) lbib_last_error(h, buf, sizeof buf, &index);
    std::ostringstream m;
    m << what << ": error " << rc << (buf[0] ? std::string(": ") + buf : std::string());
    if (index >= 0) m << " (index " << index << ")";
    throw UtilLib::Exception(m.str());
}

// The simulation that reporters write from: the one a SimulationRunner is
// stepping or reporting on this thread.
thread_local lbib_handle* g_active = nullptr;

struct ActiveScope {
    lbib_handle* saved;
    explicit ActiveScope(lbib_handle* h) : saved(g_active) { g_active = h; }
    ~ActiveScope() { g_active = saved; }
};

}  // namespace

// ---------------------------------------------------------------------------
// Parameters (GlobalSimulationParameters.cpp:34-97)

GlobalSimulationParameters_::GlobalSimulationParameters_()
    : currentIteration_(0), iterations_(0), reportSteps_(1), sizeX_(0), sizeY_(0), tauFluid_(1.0) {}

void GlobalSimulationParameters_::loadGlobalSimulationParameters(const std::string& fileName) {
    std::ifstream in(fileName);
    if (!in.is_open()) lbm_fail("Cannot find the parameter file.");
    file_ = fileName;
    cdeSolvers_.clear();
    std::string line;
    while (std::getline(in, line)) {
        if (line.empty() || line[0] == '#') continue;
        std::stringstream ls(line);
        std::string key;
        ls >> key;
        if (key == "CurrentIterations:") ls >> currentIteration_;
        else if (key == "Iterations:") ls >> iterations_;
        else if (key == "ReportStep:") ls >> reportSteps_;
        else if (key == "SizeX:") ls >> sizeX_;
        else if (key == "SizeY:") ls >> sizeY_;
        else if (key == "tauFluid:") ls >> tauFluid_;
        else if (key == "CDESolvers:") {
            std::string name;
            double tau;
            while (ls >> name >> tau) cdeSolvers_[name] = tau;
        }
    }
}

void GlobalSimulationParameters_::writeGlobalSimulationParameters(const std::string& fileName) const {
    std::ofstream out(fileName);
    if (!out.is_open()) lbm_fail("Cannot open the output file for the global simulation parameters.");
    out << std::setprecision(17);
    out << "#Global Parameter file\n";
    out << "CurrentIterations:\t" << currentIteration_ << "\n";
    out << "Iterations:\t" << iterations_ << "\n";
    out << "ReportStep:\t" << reportSteps_ << "\n";
    out << "SizeX:\t" << sizeX_ << "\n";
    out << "SizeY:\t" << sizeY_ << "\n";
    out << "tauFluid:\t" << tauFluid_ << "\n";
    out << "CDESolvers:";
    for (const auto& kv : cdeSolvers_) out << "\t" << kv.first << "\t" << kv.second;
    out << "\n";
}

void GlobalSimulationParameters_::printParameters() const {
    std::stringstream m;
    m << "Global simulation parameters: CurrentIterations " << currentIteration_ << ", Iterations " << iterations_
      << ", ReportStep " << reportSteps_ << ", SizeX " << sizeX_ << ", SizeY " << sizeY_ << ", tauFluid "
      << tauFluid_ << ", CDESolvers";
    for (const auto& kv : cdeSolvers_) m << " " << kv.first << " (tau " << kv.second << ")";
    LOG(UtilLib::logINFO) << m.str();
}

// ---------------------------------------------------------------------------
// GeometryNode

namespace nodes {

void GeometryNode::setPos(double x, double y) {
    pos_ = Field<double>(x, y);
    if (owner_) owner_->markEdited();
}

unsigned int GeometryNode::getDomainIdOfAdjacentConnections() const {
    if (connections_[0]) return connections_[0]->getDomainIdentifier();
    if (connections_[1]) return connections_[1]->getDomainIdentifier();
    return 0;
}

}  // namespace nodes

// ---------------------------------------------------------------------------
// Geometry

namespace geometry {

Geometry::Geometry(const std::string& filename) : file_(filename), h_(nullptr), stale_(false), edited_(false) {
    load(filename);
}

Geometry::~Geometry() {}

std::shared_ptr<nodes::GeometryNode> Geometry::mirrorNode(unsigned int id, double x, double y) const {
    std::shared_ptr<nodes::GeometryNode> n = std::make_shared<nodes::GeometryNode>(x, y, id);
    n->setOwner(const_cast<Geometry*>(this));
    return n;
}

// Geometry::loadGeometryTXT (Geometry.cpp:99-160), or a .vtm written by the
// cell reporter (Geometry::loadGeometryVTK, Geometry.cpp:162-306, read by
// the device runtime's parser).  The positions are the file's; the device
// perturbs them as GeometryNode's constructor does when the simulation is built.
void Geometry::load(const std::string& filename) {
    const bool vtm = filename.size() > 4 && filename.compare(filename.size() - 4, 4, ".vtm") == 0;
    if (vtm) {
        int counts[2] = {0, 0};
        if (lbib_read_vtm_geometry(filename.c_str(), nullptr, nullptr, 0, nullptr, 0, counts) != LBIB_OK)
            lbm_fail("Cannot read the geometry file " + filename);
        std::vector<unsigned> ids(counts[0]), conns(3 * (size_t)counts[1]);
        std::vector<double> xy(2 * (size_t)counts[0]);
        if (lbib_read_vtm_geometry(filename.c_str(), ids.data(), xy.data(), counts[0], conns.data(), counts[1],
                                   counts) != LBIB_OK)
            lbm_fail("Cannot read the geometry file " + filename);
        for (int i = 0; i < counts[0]; ++i) nodes_[ids[i]] = mirrorNode(ids[i], xy[2 * i], xy[2 * i + 1]);
        for (int c = 0; c < counts[1]; ++c) {
            auto a = nodes_.at(conns[3 * c]), b = nodes_.at(conns[3 * c + 1]);
            connections_.push_back(std::make_shared<Connection>(a, b, Connection::Descriptor(), conns[3 * c + 2]));
            a->setConnection<1>(connections_.back());
            b->setConnection<0>(connections_.back());
        }
        return;
    }
    std::ifstream in(filename);
    if (!in.is_open()) lbm_fail("Cannot find the geometry.txt file.");
    std::string line;
    bool readingNodes = true;
    while (std::getline(in, line)) {
        if (line.find("#Connection") != std::string::npos) readingNodes = false;
        if (line.empty() || line[0] == '#') continue;
        std::stringstream ls(line);
        if (readingNodes) {
            unsigned id;
            double x, y;
            ls >> id >> x >> y;
            nodes_[id] = mirrorNode(id, x, y);
        } else {
            unsigned a, b, d;
            ls >> a >> b >> d;
            Connection::Descriptor desc;
            std::string s1, s2;
            while (ls >> s1 >> s2) desc[s1].push_back(s2);
            connections_.push_back(std::make_shared<Connection>(nodes_.at(a), nodes_.at(b), desc, d));
            nodes_.at(a)->setConnection<1>(connections_.back());
            nodes_.at(b)->setConnection<0>(connections_.back());
            descriptors_[std::make_pair(a, b)] = desc;
        }
    }
}

void Geometry::attach(lbib_handle* h) const {
    h_ = h;
    stale_ = h != nullptr;
}

// The device's nodes and connections into the mirror; node objects keep
// their identity across refreshes.
void Geometry::refresh() const {
    if (!stale_ || !h_) return;
    stale_ = false;
    long long sz[10];
    check(h_, lbib_get_sizes(h_, sz), "lbib_get_sizes");
    const size_t M = (size_t)sz[3], C = (size_t)sz[4];
    std::vector<unsigned> ids(M), conns(3 * C);
    std::vector<double> state(6 * M);
    check(h_, lbib_download_membrane(h_, ids.data(), state.data()), "lbib_download_membrane");
    check(h_, lbib_download_connections(h_, conns.data()), "lbib_download_connections");
    std::map<unsigned int, std::shared_ptr<nodes::GeometryNode>> next;
    for (size_t i = 0; i < M; ++i) {
        auto it = nodes_.find(ids[i]);
        std::shared_ptr<nodes::GeometryNode> n = it != nodes_.end() ? it->second : mirrorNode(ids[i], 0.0, 0.0);
        const double* s = &state[6 * i];
        n->mirrorState(s[0], s[1], s[2], s[3], s[4], s[5]);
        n->setConnection<0>(nullptr);
        n->setConnection<1>(nullptr);
        next[ids[i]] = n;
    }
    nodes_.swap(next);
    connections_.clear();
    for (size_t c = 0; c < C; ++c) {
        auto a = nodes_.at(conns[3 * c]), b = nodes_.at(conns[3 * c + 1]);
        auto d = descriptors_.find(std::make_pair(conns[3 * c], conns[3 * c + 1]));
        connections_.push_back(std::make_shared<Connection>(
            a, b, d != descriptors_.end() ? d->second : Connection::Descriptor(), conns[3 * c + 2]));
        a->setConnection<1>(connections_.back());
        b->setConnection<0>(connections_.back());
    }
}

const std::map<unsigned int, std::shared_ptr<nodes::GeometryNode>>& Geometry::getGeometryNodes() const {
    refresh();
    return nodes_;
}

const std::vector<std::shared_ptr<Connection>>& Geometry::getConnections() const {
    refresh();
    return connections_;
}

void Geometry::writeGeometry(const std::string& fileName) const {
    refresh();
    std::ofstream out(fileName);
    if (!out.is_open()) lbm_fail("Cannot open the output file for the geometry.");
    out << std::setprecision(17);
    out << "#Nodes (id\txPos\tyPos)\n";
    for (const auto& kv : nodes_) out << kv.first << "\t" << kv.second->getXPos() << "\t" << kv.second->getYPos() << "\n";
    out << "#Connection (nodeId1\tnodeId2\tdomainId\tbsolver\tcdesolver\t...)\n";
    for (const auto& c : connections_) {
        out << c->getGeometryNodes().first->getId() << "\t" << c->getGeometryNodes().second->getId() << "\t"
            << c->getDomainIdentifier();
        for (const auto& kv : c->getBoundaryConditionDescriptor())
            for (const auto& v : kv.second) out << "\t" << kv.first << "\t" << v;
        out << "\n";
    }
}

const std::vector<std::shared_ptr<nodes::GeometryNode>> Geometry::getGeometryNodesWithinRadius(
    const double x, const double y, const double radius) const {
    if (!h_) lbm_fail("range queries need a running simulation");
    refresh();
    std::vector<unsigned> ids(4096);
    int n = lbib_nodes_within_radius(h_, x, y, radius, -1, ids.data(), (int)ids.size());
    if (n > (int)ids.size()) {
        ids.resize(n);
        n = lbib_nodes_within_radius(h_, x, y, radius, -1, ids.data(), (int)ids.size());
    }
    if (n < 0) check(h_, -n, "lbib_nodes_within_radius");
    std::vector<std::shared_ptr<nodes::GeometryNode>> out;
    for (int i = 0; i < n; ++i) out.push_back(nodes_.at(ids[i]));
    return out;
}

const std::vector<std::shared_ptr<nodes::GeometryNode>> Geometry::getGeometryNodesWithinRadiusWithAvoidance(
    const double x, const double y, const double radius, const unsigned int domainIdentifier) const {
    if (!h_) lbm_fail("range queries need a running simulation");
    refresh();
    std::vector<unsigned> ids(4096);
    int n = lbib_nodes_within_radius(h_, x, y, radius, (long long)domainIdentifier, ids.data(), (int)ids.size());
    if (n > (int)ids.size()) {
        ids.resize(n);
        n = lbib_nodes_within_radius(h_, x, y, radius, (long long)domainIdentifier, ids.data(), (int)ids.size());
    }
    if (n < 0) check(h_, -n, "lbib_nodes_within_radius");
    std::vector<std::shared_ptr<nodes::GeometryNode>> out;
    for (int i = 0; i < n; ++i) out.push_back(nodes_.at(ids[i]));
    return out;
}

std::shared_ptr<nodes::GeometryNode> Geometry::getGeometryNodesWithinRadiusWithAvoidanceClosest(
    const double x, const double y, const double radius, const unsigned int domainIdentifier) const {
    if (!h_) lbm_fail("range queries need a running simulation");
    refresh();
    const long long avoid = (long long)domainIdentifier;
    long long closest = -1;
    check(h_, lbib_closest_nodes(h_, &x, &y, &avoid, 1, radius, &closest), "lbib_closest_nodes");
    if (closest < 0) return nullptr;
    return nodes_.at((unsigned)closest);
}

unsigned int Geometry::addGeometryNode(const double x, const double y) {
    refresh();
    const unsigned id = nodes_.empty() ? 0u : nodes_.rbegin()->first + 1;
    nodes_[id] = mirrorNode(id, x, y);
    edited_ = true;
    return id;
}

unsigned int Geometry::removeGeometryNode(const unsigned int nodeid) {
    refresh();
    edited_ = true;
    return (unsigned)nodes_.erase(nodeid);
}

void Geometry::eraseConnection(std::shared_ptr<Connection> toDelete) {
    refresh();
    auto it = std::find(connections_.begin(), connections_.end(), toDelete);
    if (it == connections_.end()) lbm_fail("eraseConnection: no such connection");
    connections_.erase(it);
    edited_ = true;
}

void Geometry::addConnection(std::shared_ptr<nodes::GeometryNode> p1, std::shared_ptr<nodes::GeometryNode> p2,
                             const std::map<std::string, std::vector<std::string>>& descriptor,
                             const unsigned int domainIdentifier) {
    refresh();
    connections_.push_back(std::make_shared<Connection>(p1, p2, descriptor, domainIdentifier));
    p1->setConnection<1>(connections_.back());
    p2->setConnection<0>(connections_.back());
    descriptors_[std::make_pair(p1->getId(), p2->getId())] = descriptor;
    edited_ = true;
}

bool Geometry::checkGeometryIntegrity() const {
    refresh();
    std::map<unsigned, int> in, out;
    for (const auto& c : connections_) {
        out[c->getGeometryNodes().first->getId()]++;
        in[c->getGeometryNodes().second->getId()]++;
    }
    for (const auto& kv : nodes_)
        if (in[kv.first] != 1 || out[kv.first] != 1) return false;
    return true;
}

std::map<unsigned int, unsigned int> Geometry::getCellTypeTrackerMap(void) const {
    refresh();
    std::map<unsigned int, unsigned int> m;
    m[0] = 0;
    for (const auto& c : connections_) m[c->getDomainIdentifier()] = 1;
    return m;
}

// Geometry::addGeometryNode / removeGeometryNode / addConnection /
// eraseConnection on the device: the resulting lists (lbib_upload_membrane).
void Geometry::pushEdits() const {
    if (!edited_ || !h_) return;
    std::vector<unsigned> ids, conns;
    std::vector<double> xy;
    for (const auto& kv : nodes_) {
        ids.push_back(kv.first);
        xy.push_back(kv.second->getXPos());
        xy.push_back(kv.second->getYPos());
    }
    for (const auto& c : connections_) {
        conns.push_back(c->getGeometryNodes().first->getId());
        conns.push_back(c->getGeometryNodes().second->getId());
        conns.push_back(c->getDomainIdentifier());
    }
    check(h_, lbib_upload_membrane(h_, ids.data(), xy.data(), (int)ids.size(), conns.data(),
                                   (int)(conns.size() / 3)),
          "lbib_upload_membrane");
    edited_ = false;
    stale_ = true;
}

// ---------------------------------------------------------------------------
// GeometryHandler and the lattice views

struct GeometryHandler::Snapshot {
    bool valid = false;
    int nx = 0, ny = 0, S = 0;
    std::vector<double> f, g, vel;
    std::vector<unsigned> dom, ctype;
};

GeometryHandler::GeometryHandler(const Geometry& geometry)
    : geometry_(geometry), h_(nullptr), cellTypesSet_(false), snap_(std::make_shared<Snapshot>()) {
    cellTypes_ = geometry.getCellTypeTrackerMap();
}

GeometryHandler::~GeometryHandler() {}

void GeometryHandler::attach(lbib_handle* h) {
    h_ = h;
    geometry_.attach(h);
    invalidate();
    // cell types the application set before the simulation was built
    if (h_ && cellTypesSet_) copyCellTypeToPhysicalNodes(cellTypes_);
}

void GeometryHandler::invalidate() const {
    snap_->valid = false;
    geometry_.invalidate();
}

const std::vector<std::vector<nodes::PhysicalNode*>>& GeometryHandler::getPhysicalNodes() const {
    const int nx = (int)Parameters.getSizeX(), ny = (int)Parameters.getSizeY();
    if ((int)grid_.size() != ny || (ny > 0 && (int)grid_[0].size() != nx)) {
        views_.clear();
        views_.reserve((size_t)nx * ny);
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) views_.emplace_back(x, y, this);
        grid_.assign(ny, std::vector<nodes::PhysicalNode*>(nx, nullptr));
        for (int y = 0; y < ny; ++y)
            for (int x = 0; x < nx; ++x) grid_[y][x] = &views_[(size_t)y * nx + x];
    }
    return grid_;
}

const GeometryHandler::Snapshot& GeometryHandler::snapshot() const {
    if (snap_->valid) return *snap_;
    if (!h_) lbm_fail("the lattice is on the device: it exists once the simulation is built (initSolvers)");
    long long sz[10];
    check(h_, lbib_get_sizes(h_, sz), "lbib_get_sizes");
    Snapshot& s = *snap_;
    s.nx = (int)sz[0];
    s.ny = (int)sz[1];
    s.S = (int)sz[2];
    const size_t L = (size_t)s.nx * s.ny;
    s.f.resize(9 * L);
    s.g.resize(5 * L * (size_t)std::max(1, s.S));
    s.vel.resize(2 * L);
    s.dom.resize(L);
    s.ctype.resize(L);
    check(h_, lbib_download_lattice(h_, s.f.data(), s.S ? s.g.data() : nullptr, s.vel.data(), nullptr, s.dom.data(),
                                    s.ctype.data()),
          "lbib_download_lattice");
    s.valid = true;
    return s;
}

int GeometryHandler::species(const std::string& name) const {
    int k = 0;
    for (const auto& kv : Parameters.getCdeSolvers()) {
        if (kv.first == name) return k;
        ++k;
    }
    lbm_fail("no CDE solver named " + name);
    return -1;
}

const std::map<unsigned int, double> GeometryHandler::computeAreas() const {
    std::map<unsigned int, double> out;
    if (!h_) lbm_fail("computeAreas needs a running simulation");
    geometry_.pushEdits();
    int n = lbib_areas(h_, nullptr, nullptr, 0);
    if (n < 0) check(h_, -n, "lbib_areas");
    std::vector<unsigned> dom(n);
    std::vector<double> area(n);
    n = lbib_areas(h_, dom.data(), area.data(), n);
    if (n < 0) check(h_, -n, "lbib_areas");
    for (int i = 0; i < n; ++i) out[dom[i]] = area[i];
    return out;
}

std::map<unsigned int, double> GeometryHandler::computeAccumulatedDomainConcentrations(const std::string& name) const {
    std::map<unsigned int, double> out;
    if (!h_) lbm_fail("computeAccumulatedDomainConcentrations needs a running simulation");
    int nd = 0;
    check(h_, lbib_get_domain_count(h_, &nd), "lbib_get_domain_count");
    std::vector<unsigned> dom(nd + 1);
    std::vector<double> acc(nd + 1);
    const int n = lbib_accumulated_concentrations(h_, name.c_str(), dom.data(), acc.data(), nd + 1);
    if (n < 0) check(h_, -n, "lbib_accumulated_concentrations");
    for (int i = 0; i < n; ++i) out[dom[i]] = acc[i];
    return out;
}

void GeometryHandler::cureLattice() {
    if (!h_) return;
    geometry_.pushEdits();
    check(h_, lbib_cure_lattice(h_), "lbib_cure_lattice");
    invalidate();
}

unsigned int GeometryHandler::createGeometryNode(const double xpos, const double ypos) {
    return const_cast<Geometry&>(geometry_).addGeometryNode(xpos, ypos);
}

void GeometryHandler::createConnection(std::shared_ptr<nodes::GeometryNode> const p1,
                                       std::shared_ptr<nodes::GeometryNode> const p2,
                                       const std::map<std::string, std::vector<std::string>> boundaryconditiondescriptor,
                                       const unsigned int domainidentifier) {
    const_cast<Geometry&>(geometry_).addConnection(p1, p2, boundaryconditiondescriptor, domainidentifier);
}

void GeometryHandler::eraseConnection(std::shared_ptr<Connection> toErase) {
    const_cast<Geometry&>(geometry_).eraseConnection(toErase);
}

const std::shared_ptr<nodes::GeometryNode> GeometryHandler::returnGeometryNode(const unsigned int nodeID) const {
    const auto& n = geometry_.getGeometryNodes();
    auto it = n.find(nodeID);
    if (it == n.end()) lbm_fail("returnGeometryNode: no node with that id");
    return it->second;
}

// The device's cell-type table for domain 0 and the domains of the
// connections (the reference's map holds exactly those).
std::map<unsigned int, unsigned int>& GeometryHandler::getCellTypeTrackerMap() {
    if (h_) {
        int nd = 0;
        check(h_, lbib_get_domain_count(h_, &nd), "lbib_get_domain_count");
        std::vector<unsigned> dom(nd), type(nd);
        const int n = lbib_get_cell_types(h_, dom.data(), type.data(), nd);
        if (n < 0) check(h_, -n, "lbib_get_cell_types");
        std::set<unsigned> present;
        present.insert(0u);
        for (const auto& c : geometry_.getConnections()) present.insert(c->getDomainIdentifier());
        cellTypes_.clear();
        for (int i = 0; i < n; ++i)
            if (present.count(dom[i])) cellTypes_[dom[i]] = type[i];
    }
    return cellTypes_;
}

void GeometryHandler::copyCellTypeToPhysicalNodes(std::map<unsigned int, unsigned int>& celltrackermap) {
    if (&celltrackermap != &cellTypes_) cellTypes_ = celltrackermap;
    cellTypesSet_ = true;
    if (!h_) return;
    std::vector<unsigned> dom, type;
    for (const auto& kv : celltrackermap) {
        dom.push_back(kv.first);
        type.push_back(kv.second);
    }
    check(h_, lbib_set_cell_types(h_, dom.data(), type.data(), (int)dom.size()), "lbib_set_cell_types");
    snap_->valid = false;
}

void GeometryHandler::copyCellTypeToPhysicalNodes(unsigned int domainidentifier, unsigned int celltype) {
    cellTypes_[domainidentifier] = celltype;
    cellTypesSet_ = true;
    if (!h_) return;
    check(h_, lbib_set_cell_types(h_, &domainidentifier, &celltype, 1), "lbib_set_cell_types");
    snap_->valid = false;
}

}  // namespace geometry

namespace nodes {

namespace {
size_t node_index(const PhysicalNode& n, const geometry::GeometryHandler::Snapshot& s) {
    return (size_t)n.getYPos() * s.nx + n.getXPos();
}
}  // namespace

unsigned int PhysicalNode::getDomainIdentifier() const {
    const auto& s = owner_->snapshot();
    return s.dom[node_index(*this, s)];
}

unsigned int PhysicalNode::getCellType() const {
    const auto& s = owner_->snapshot();
    return s.ctype[node_index(*this, s)];
}

CDESolverView PhysicalNode::getCDESolverSlow(const std::string& name) const {
    return CDESolverView(*this, owner_->species(name));
}

Field<double> FluidSolverView::getVelocity() const {
    const auto& s = node_.owner()->snapshot();
    const size_t n = node_index(node_, s);
    return Field<double>(s.vel[2 * n], s.vel[2 * n + 1]);
}

// FluidSolver::getRho: the sum of the nine distributions in slot order
double FluidSolverView::getRho() const {
    const auto& s = node_.owner()->snapshot();
    const size_t n = node_index(node_, s);
    double r = 0.0;
    for (int d = 0; d < 9; ++d) r += s.f[9 * n + d];
    return r;
}

void FluidSolverView::addMass(double) {
    lbm_fail("FluidSolver::addMass has no host path here: the mass sources are the device bio solvers' "
             "(LbibAreaRegulator, the tutorial area regulator, the growth solvers)");
}

// CDESolverD2Q5::getC: the sum of the five distributions in slot order
double CDESolverView::getC() const {
    const auto& s = node_.owner()->snapshot();
    const size_t L = (size_t)s.nx * s.ny;
    const size_t n = node_index(node_, s);
    double c = 0.0;
    for (int d = 0; d < 5; ++d) c += s.g[((size_t)k_ * L + n) * 5 + d];
    return c;
}

}  // namespace nodes

// ---------------------------------------------------------------------------
// ForceSolver

namespace solver {

// ForceSolver::addForce's record formats (ForceStructs.hpp): the number of
// node ids and parameters each type reads.
void ForceSolver::addForce(std::stringstream* const forcedescriptor) {
    int type = -1;
    (*forcedescriptor) >> type;
    unsigned id1 = 0, id2 = 0;
    double p[4] = {0, 0, 0, 0};
    int np = 0;
    (*forcedescriptor) >> id1;
    switch (type) {
        case 0: case 7: (*forcedescriptor) >> id2; np = 2; break;
        case 1: np = 4; break;
        case 2: np = 2; break;
        case 3: case 4: np = 3; break;
        case 5: case 6: (*forcedescriptor) >> id2; np = 1; break;
        default: lbm_fail("ForceSolver::addForce: unknown force type");
    }
    for (int i = 0; i < np; ++i) (*forcedescriptor) >> p[i];
    if (forcedescriptor->fail()) lbm_fail("ForceSolver::addForce: malformed force record");
    type_.push_back(type);
    id1_.push_back(id1);
    id2_.push_back(id2);
    par_.insert(par_.end(), p, p + 4);
    if (!h_) lbm_fail("ForceSolver::addForce needs a running simulation (load static forces with initForceSolver)");
}

void ForceSolver::flush() {
    if (type_.empty() || !h_) return;
    const int rc = lbib_add_forces(h_, type_.data(), id1_.data(), id2_.data(), par_.data(), (int)type_.size());
    type_.clear();
    id1_.clear();
    id2_.clear();
    par_.clear();
    check(h_, rc, "lbib_add_forces");
}

void ForceSolver::deleteAllForces() {
    if (!h_) return;
    flush();
    check(h_, lbib_delete_all_forces(h_), "lbib_delete_all_forces");
}

void ForceSolver::deleteForceType(const unsigned int forcetype) {
    if (!h_) return;
    flush();
    check(h_, lbib_delete_force_type(h_, (int)forcetype), "lbib_delete_force_type");
}

void ForceSolver::writeForceSolver(const std::string& filename) const {
    if (!h_) lbm_fail("writeForceSolver needs a running simulation");
    const_cast<ForceSolver*>(this)->flush();
    check(h_, lbib_write_simulation(h_, filename.c_str(), nullptr, nullptr, nullptr), "lbib_write_simulation");
}

}  // namespace solver

// ---------------------------------------------------------------------------
// Reporters

namespace reportHandler {

void writeVtkBlock(const std::string& filename, unsigned int time, int kind, unsigned int coarsening) {
    if (!g_active) return;
    check(g_active, lbib_write_vtk(g_active, filename.c_str(), time, kind, (int)(coarsening ? coarsening : 1)),
          "lbib_write_vtk");
}

}  // namespace reportHandler

// ---------------------------------------------------------------------------
// SimulationRunner

namespace {

// The names the device runtime runs itself (load_plugins in lbib_host.cu).
bool device_bio_solver(const std::string& n) {
    static const std::set<std::string> names = {
        "LbibMembraneTension", "tutorial_01_BioSolverMembraneTension", "tutorial_02_BioSolverMembraneTension",
        "BioSolverMembraneTension", "tutorial_01_BioSolverAreaRegulator", "LbibAreaRegulator",
        "tutorial_01_BioSolverDifferentiation", "BioSolverDifferentiation", "tutorial_02_BioSolverGrowth",
        "BioSolverGrowth", "BioSolverEmpty", "tutorial_01_BioSolverCellJunction", "tutorial_02_BioSolverCellJunction",
        "BioSolverCellJunction", "LbibCellJunction", "tutorial_01_BioSolverCellDivision",
        "tutorial_02_BioSolverCellDivision", "BioSolverCellDivision", "LbibCellDivision"};
    return names.count(n) != 0;
}

}  // namespace

SimulationRunner::SimulationRunner(const geometry::GeometryHandler& geometry,
                                   const reportHandler::ReportHandler& reportHandler)
    : geometryHandler_(const_cast<geometry::GeometryHandler&>(geometry)),
      reportHandler_(reportHandler),
      h_(nullptr),
      configChanged_(false),
      velocityInit_(false) {}

SimulationRunner::~SimulationRunner() {
    if (h_) {
        geometryHandler_.attach(nullptr);
        lbib_destroy(h_);
    }
}

lbib_handle* SimulationRunner::deviceHandle() {
    requireDevice();
    return h_;
}

// Builds the device simulation from the parameter file (as loaded, with the
// current iteration), the geometry (its file, or the mirror once a plugin
// edited it), the force file and the registered device solvers, then replays
// what was done to the lattice before.
void SimulationRunner::build() {
    if (workDir_.empty()) {
        char tmpl[] = "/tmp/lbibcell_dropin_XXXXXX";
        if (!mkdtemp(tmpl)) lbm_fail("cannot create a working directory");
        workDir_ = tmpl;
    }
    const std::string params = workDir_ + "/parameters.txt";
    Parameters.writeGlobalSimulationParameters(params);
    std::string geom = geometryHandler_.getGeometry().sourceFile();
    if (geometryHandler_.getGeometry().edited()) {
        geom = workDir_ + "/geometry.txt";
        geometryHandler_.getGeometry().writeGeometry(geom);
    }
    const std::string plugins = workDir_ + "/plugins.txt";
    {
        // The reference's own solvers take no parameters; the configuration
        // plugins (LbibMembraneTension, LbibAreaRegulator, the Lbib species, a
        // force model) read theirs from a plugin file (format:
        // lbibcell_b200/configs.py) named by LBIB_PLUGIN_FILE: its lines for the
        // registered bio solvers give their parameters, and its CDE,
        // CDESource and ForceModel lines are taken as they are.
        std::map<std::string, std::string> bioLine;
        std::vector<std::string> other;
        if (const char* pf = std::getenv("LBIB_PLUGIN_FILE")) {
            std::ifstream in(pf);
            if (!in.is_open()) lbm_fail(std::string("Cannot find the plugin file ") + pf);
            std::string line;
            while (std::getline(in, line)) {
                std::stringstream ls(line);
                std::string kind, name;
                ls >> kind >> name;
                if (kind == "BioSolver") bioLine[name] = line;
                else if (kind == "CDE" || kind == "CDESource" || kind == "ForceModel") other.push_back(line);
            }
        }
        std::ofstream out(plugins);
        out << "#plugins of the application\n";
        for (const auto& m : massSolvers_) out << "MassSolver\t" << m << "\n";
        for (const auto& b : deviceBio_)
            out << (bioLine.count(b) ? bioLine[b] : "BioSolver\t" + b) << "\n";
        for (const auto& l : other) out << l << "\n";
    }
    const char* prec = std::getenv("LBIB_PRECISION");
    const int precision = (prec && std::string(prec) == "fp32") ? LBIB_FP32_SHIFTED : LBIB_FP64;
    const char* dev = std::getenv("LBIB_DEVICE");
    if (h_) {
        geometryHandler_.attach(nullptr);
        forceSolver_.attach(nullptr);
        lbib_destroy(h_);
        h_ = nullptr;
    }
    lbib_handle* h = nullptr;
    const int rc = lbib_create_from_files(params.c_str(), geom.c_str(), forceSolver_.forceFile().c_str(),
                                          plugins.c_str(), precision, dev ? std::atoi(dev) : 0, &h);
    if (rc != LBIB_OK) {
        std::string msg = "building the device simulation failed: error " + std::to_string(rc);
        if (h) {
            char buf[512] = {0};
            lbib_last_error(h, buf, sizeof buf, nullptr);
            msg += std::string(": ") + buf;
            lbib_destroy(h);
        }
        throw UtilLib::Exception(msg);
    }
    h_ = h;
    geometryHandler_.attach(h_);
    forceSolver_.attach(h_);
    configChanged_ = false;
    if (velocityInit_) check(h_, lbib_init_velocity(h_, velocity_.x, velocity_.y), "lbib_init_velocity");
    if (!restartFile_.empty()) check(h_, lbib_load_solvers(h_, restartFile_.c_str()), "lbib_load_solvers");
    geometryHandler_.invalidate();
}

void SimulationRunner::requireDevice() {
    if (!h_ || configChanged_) build();
}

void SimulationRunner::initSolvers() {
    requireDevice();
    ActiveScope scope(h_);
    reportHandler_.writeReport(0);
}

void SimulationRunner::initSolvers(Field<double> fluidVelocity) {
    velocityInit_ = true;
    velocity_ = fluidVelocity;
    restartFile_.clear();
    if (h_ && !configChanged_) check(h_, lbib_init_velocity(h_, velocity_.x, velocity_.y), "lbib_init_velocity");
    geometryHandler_.invalidate();
}

void SimulationRunner::initSolvers(const std::string& filename) {
    restartFile_ = filename;
    if (h_ && !configChanged_) check(h_, lbib_load_solvers(h_, filename.c_str()), "lbib_load_solvers");
    geometryHandler_.invalidate();
}

void SimulationRunner::initForceSolver(const std::string& fileName) {
    forceSolver_.loadForceFile(fileName);
    configChanged_ = true;
}

void SimulationRunner::addMassSolver(const std::string& name) {
    if (name != "MassSolverBoxOutlet") throw std::bad_typeid();
    massSolvers_.push_back(name);
    configChanged_ = true;
}

void SimulationRunner::addBioSolver(const std::string& name) {
    if (solver::BioSolverFactory::instance().isRegistered(name)) {
        hostBio_.emplace_back(solver::BioSolverFactory::instance().createObject(name));
        return;
    }
    if (!device_bio_solver(name)) throw std::bad_typeid();
    if (!hostBio_.empty())
        lbm_fail("bio solver " + name + " runs on the device, inside the step: register it before the host plugins");
    deviceBio_.push_back(name);
    configChanged_ = true;
}

void SimulationRunner::stepDevice(unsigned int n) {
    if (n == 0) return;
    const int rc = lbib_step(h_, (int)n);
    geometryHandler_.invalidate();
    check(h_, rc, "lbib_step");
}

// The host plugins of the step just run, in registration order; their
// geometry and force edits reach the device before the next step.
void SimulationRunner::runHostBio() {
    for (auto& b : hostBio_) {
        b->applyBioProcess(geometryHandler_, forceSolver_);
        forceSolver_.flush();
        geometryHandler_.getGeometry().pushEdits();
        geometryHandler_.invalidate();
    }
}

void SimulationRunner::runSimulation() {
    unsigned int t = 0;
    try {
        requireDevice();
        ActiveScope scope(h_);
        const unsigned int total = Parameters.getIterations();
        const unsigned int every = std::max(1u, Parameters.getReportSteps());
        t = 1;
        while (t <= total) {
            // without host plugins, the device runs up to the next report in one call
            unsigned int n = 1;
            if (hostBio_.empty()) {
                const unsigned int nextReport = ((t + every - 1) / every) * every;
                n = std::min(total, nextReport) - t + 1;
            }
            stepDevice(n);
            if (!hostBio_.empty()) runHostBio();
            for (unsigned int k = 0; k < n; ++k) Parameters++;
            t += n;
            reportHandler_.writeReport(t - 1);
        }
    } catch (const std::exception& exp) {
        // SimulationRunner.cpp:101-109: report everything, dump the state,
        // print the error.  A device error leaves the handle refusing work, so
        // the crash reports write what they can and their own failures are
        // not reported over the original error.
        Parameters.setReportSteps(1);
        if (h_) {
            ActiveScope scope(h_);
            try {
                reportHandler_.writeCrashReport(t);
            } catch (const std::exception&) {
            }
            const std::string s = std::to_string(t);
            lbib_write_simulation(h_, ("output/CRASH_forceOut_" + s + ".txt").c_str(),
                                  ("output/CRASH_geoOut_" + s + ".txt").c_str(),
                                  ("output/CRASH_parameterOut_" + s + ".txt").c_str(),
                                  ("output/CRASH_solverOut_" + s + ".txt").c_str());
        }
        std::cout << exp.what() << std::endl;
    }
}

void SimulationRunner::writeSimulation(const std::string& forceFileName, const std::string& geometryFileName,
                                       const std::string& parameterFileName, const std::string& solverFileName) {
    requireDevice();
    forceSolver_.flush();
    check(h_, lbib_write_simulation(h_, forceFileName.c_str(), geometryFileName.c_str(), parameterFileName.c_str(),
                                    solverFileName.c_str()),
          "lbib_write_simulation");
}

}  // namespace LbmLib
