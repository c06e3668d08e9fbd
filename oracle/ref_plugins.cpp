// ref_plugins.cpp — the lbibcell_b200 configuration plugins, written against
// the reference's own plugin API so that they self-register in the
// reference build (oracle/_ref).  TEST INFRASTRUCTURE ONLY.
//
// The reference hard-codes its physics constants inside each plugin
// (e.g. libs/LbmLib/src/solver/BioSolver/tutorial_01_BioSolverMembraneTension.cpp:33-36).
// These plugins take theirs from the plugin file instead (format documented
// in lbibcell_b200/configs.py), filled in by ref_driver.cpp through
// lbibref::registry() before the simulation is built.
//
//   LbibMembraneTension   type-6 tension pair on every connection, renewed
//                         every `frequency` iterations (as tutorial_01's).
//   LbibAreaRegulator     per-cell mass source strength*(target-A)/target,
//                         clamped to +-maxsource, target = factor * first A.
//   LbibCellJunction      the cell-junction solver of tutorial_01 (every 10th
//                         iteration: drop type-7 forces, then for each node in
//                         id order a type-7 spring each way to the closest node
//                         of another cell within `radius`) with radius, spring
//                         constant k and rest length l0 from the plugin file.
//   LbibCellDivision      every `frequency` iterations, a cell whose area
//                         exceeds `factor` times its reference area (its area
//                         when this solver first saw it; a daughter inherits
//                         its mother's) splits across the perpendicular
//                         bisector of its longest axis, as tutorial_01's
//                         division does; then the lattice is cured.
//   LbibCDESolverD2Q5_A/B/C  D2Q5 species with R = source[domain] - decay*C,
//                         added as dt*R/3 (rest) and dt*R/6 (moving) like
//                         tutorial_01_CDESolverD2Q5_SIGNAL.cpp:102-135.

#include <LbmLib/include/GlobalSimulationParameters.hpp>
#include <LbmLib/include/geometry/GeometryHandler.hpp>
#include <LbmLib/include/nodes/BoundaryNode.hpp>
#include <LbmLib/include/nodes/GeometryNode.hpp>
#include <LbmLib/include/nodes/PhysicalNode.hpp>
#include <LbmLib/include/solver/BioSolver/BioBaseSolver.hpp>
#include <LbmLib/include/solver/CDESolver/CDEAbstractSolver.hpp>
#include <LbmLib/include/solver/FluidSolver/FluidSolver.hpp>
#include <LbmLib/include/solver/ForceSolver.hpp>
#include <LbmLib/include/geometry/Connection.hpp>

#include <array>
#include <cmath>
#include <iterator>
#include <map>
#include <numeric>
#include <sstream>
#include <string>

#include "ref_registry.hpp"

namespace lbibref {
Registry& registry() {
    static Registry r;
    return r;
}
}  // namespace lbibref

namespace LbmLib {
namespace solver {

// ---------------------------------------------------------------------------
class LbibMembraneTension : public BioBaseSolver<LbibMembraneTension> {
 public:
    LbibMembraneTension();
    virtual void applyBioProcess(geometry::GeometryHandler& gh, solver::ForceSolver& fs) {
        const auto& p = lbibref::registry().tension;
        auto conns = gh.getGeometry().getConnections();
        if (Parameters.getCurrentIteration() % p.frequency != 0) return;
        fs.deleteForceType(6);
        std::stringstream d;
        for (size_t j = 0; j < conns.size(); ++j) {
            d.str(std::string()); d.clear();
            d << "6\t" << conns[j]->getGeometryNodes().first->getId() << "\t"
              << conns[j]->getGeometryNodes().second->getId() << "\t" << p.force;
            fs.addForce(&d);
            d.str(std::string()); d.clear();
            d << "6\t" << conns[j]->getGeometryNodes().second->getId() << "\t"
              << conns[j]->getGeometryNodes().first->getId() << "\t" << p.force;
            fs.addForce(&d);
        }
    }
    static const std::string name;
};
const std::string LbibMembraneTension::name = "LbibMembraneTension";

// ---------------------------------------------------------------------------
class LbibAreaRegulator : public BioBaseSolver<LbibAreaRegulator> {
 public:
    LbibAreaRegulator();
    virtual void applyBioProcess(geometry::GeometryHandler& gh, solver::ForceSolver&) {
        const auto& p = lbibref::registry().area;
        std::map<unsigned int, double> areas = gh.computeAreas();
        for (auto it : areas)
            if (target_.find(it.first) == target_.end()) target_[it.first] = p.factor * it.second;
        std::map<unsigned int, double> src;
        for (auto it : areas) {
            const double tgt = target_[it.first];
            double r = p.strength * (tgt - it.second) / tgt;
            if (r > p.maxsource) r = p.maxsource;
            else if (r < -p.maxsource) r = -p.maxsource;
            src[it.first] = r;
        }
        const auto& grid = gh.getPhysicalNodes();
        for (size_t y = 0; y < grid.size(); ++y)
            for (size_t x = 0; x < grid[0].size(); ++x) {
                const unsigned d = grid[y][x]->getDomainIdentifier();
                if (d != 0) grid[y][x]->getFluidSolver().addMass(src[d]);
            }
    }
    static const std::string name;
 private:
    std::map<unsigned int, double> target_;
};
const std::string LbibAreaRegulator::name = "LbibAreaRegulator";

// ---------------------------------------------------------------------------
class LbibCellJunction : public BioBaseSolver<LbibCellJunction> {
 public:
    LbibCellJunction();
    virtual void applyBioProcess(geometry::GeometryHandler& gh, solver::ForceSolver& fs) {
        if (Parameters.getCurrentIteration() % 10 != 0) return;
        const auto& p = lbibref::registry().junction;
        fs.deleteForceType(7);
        const auto nodes = gh.getGeometry().getGeometryNodes();  // id order
        std::stringstream d;
        for (const auto& kv : nodes) {
            const auto& n = kv.second;
            const std::shared_ptr<nodes::GeometryNode> other =
                gh.getGeometry().getGeometryNodesWithinRadiusWithAvoidanceClosest(
                    n->getXPos(), n->getYPos(), p.radius, n->getDomainIdOfAdjacentConnections());
            if (other == nullptr) continue;
            d.str(std::string()); d.clear();
            d << "7\t" << n->getId() << "\t" << other->getId() << "\t" << p.k << "\t" << p.l0;
            fs.addForce(&d);
            d.str(std::string()); d.clear();
            d << "7\t" << other->getId() << "\t" << n->getId() << "\t" << p.k << "\t" << p.l0;
            fs.addForce(&d);
        }
    }
    static const std::string name;
};
const std::string LbibCellJunction::name = "LbibCellJunction";

// ---------------------------------------------------------------------------
class LbibCellDivision : public BioBaseSolver<LbibCellDivision> {
 public:
    LbibCellDivision();
    virtual void applyBioProcess(geometry::GeometryHandler& gh, solver::ForceSolver&) {
        const auto& p = lbibref::registry().division;
        if (Parameters.getCurrentIteration() % p.frequency != 0) return;
        auto& types = gh.getCellTypeTrackerMap();
        if (types.empty()) {
            types[0] = 0;
            for (const auto& kv : cellsOf(gh)) types[kv.first] = 1;
        }
        std::map<unsigned int, double> areas = gh.computeAreas();
        areas[0] = 0.0;
        for (const auto& a : areas)
            if (a.first != 0 && refArea_.find(a.first) == refArea_.end()) refArea_[a.first] = a.second;
        for (auto it = std::next(areas.begin()); it != areas.end(); ++it) {
            if (!(it->second > p.factor * refArea_[it->first])) continue;
            const unsigned int born = divide(gh, it->first);
            refArea_[born] = refArea_[it->first];
            types[born] = types[it->first];
            gh.cureLattice();
        }
        gh.copyCellTypeToPhysicalNodes(types);
    }
    static const std::string name;

 private:
    typedef std::shared_ptr<geometry::Connection> ConnPtr;

    // the connections of each cell, in the geometry's connection order
    static std::map<unsigned int, std::vector<ConnPtr>> cellsOf(geometry::GeometryHandler& gh) {
        std::map<unsigned int, std::vector<ConnPtr>> cells;
        for (const auto& c : gh.getGeometry().getConnections()) cells[c->getDomainIdentifier()].push_back(c);
        return cells;
    }

    // Splits cell `dom`; returns the new cell's domain id (one above the largest).
    static unsigned int divide(geometry::GeometryHandler& gh, unsigned int dom) {
        auto cells = cellsOf(gh);
        const unsigned int born = cells.rbegin()->first + 1;
        const std::vector<ConnPtr>& cell = cells[dom];
        // the two first nodes furthest apart (the first pair found of the largest distance)
        double far = 0.0;
        std::shared_ptr<nodes::GeometryNode> a, b;
        for (const auto& c1 : cell)
            for (const auto& c2 : cell) {
                const auto& p = c1->getGeometryNodes().first;
                const auto& q = c2->getGeometryNodes().first;
                const double dx = p->getXPos() - q->getXPos(), dy = p->getYPos() - q->getYPos();
                const double d = std::sqrt(dx * dx + dy * dy);
                if (d > far) { far = d; a = p; b = q; }
            }
        // the perpendicular bisector y = slope x + icpt, and the two connections it cuts
        const double mx = 0.5 * (a->getXPos() + b->getXPos()), my = 0.5 * (a->getYPos() + b->getYPos());
        const double slope = -(b->getXPos() - a->getXPos()) / (b->getYPos() - a->getYPos());
        const double icpt = my - slope * mx;
        std::vector<ConnPtr> cut;
        for (const auto& c : cell) {
            const auto& p = c->getGeometryNodes().first;
            const auto& q = c->getGeometryNodes().second;
            const bool above = p->getYPos() > slope * p->getXPos() + icpt;
            const bool below = q->getYPos() < slope * q->getXPos() + icpt;
            if (above == below) cut.push_back(c);
        }
        if (cut.size() != 2) lbm_fail("LbibCellDivision: the bisector does not cut exactly two connections");
        const auto desc = cut[0]->getBoundaryConditionDescriptor();
        if (desc != cut[1]->getBoundaryConditionDescriptor())
            lbm_fail("LbibCellDivision: the two cut connections carry different boundary solvers");
        cut[0]->getGeometryNodes().first->setConnection<1>(nullptr);
        cut[0]->getGeometryNodes().second->setConnection<0>(nullptr);
        cut[1]->getGeometryNodes().first->setConnection<1>(nullptr);
        cut[1]->getGeometryNodes().second->setConnection<0>(nullptr);
        gh.createConnection(cut[0]->getGeometryNodes().first, cut[1]->getGeometryNodes().second, desc, dom);
        gh.createConnection(cut[1]->getGeometryNodes().first, cut[0]->getGeometryNodes().second, desc, dom);
        for (const auto& c : cut) gh.eraseConnection(c);
        // the ring through the second cut's end node becomes the new cell
        const ConnPtr start = cut[1]->getGeometryNodes().second->getConnection<1>();
        ConnPtr c = start;
        do {
            c->setDomainIdentifier(born);
            c = c->getGeometryNodes().second->getConnection<1>();
        } while (c != start);
        return born;
    }

    std::map<unsigned int, double> refArea_;
};
const std::string LbibCellDivision::name = "LbibCellDivision";

// ---------------------------------------------------------------------------
template <class Self>
class LbibCDE : public BaseCDESolver<Self> {
 public:
    LbibCDE() : d_({{0.0, 0.0, 0.0, 0.0, 0.0}}) {}
    virtual ~LbibCDE() {}

    const lbibref::CdeParams& params() const { return lbibref::registry().cde[Self::name]; }

    double reaction(double C) const {
        const auto& p = params();
        auto it = p.source.find(this->physicalNode_->getDomainIdentifier());
        const double src = it == p.source.end() ? 0.0 : it->second;
        return src - p.decay * C;
    }

    virtual void initSolver() {
        for (int d = 0; d < 5; ++d) d_[d] = params().init / 5.0;
    }

    virtual void collide() {
        const double C = getC();
        const double ux = this->physicalNode_->getFluidSolver().getVelocity().x;
        const double uy = this->physicalNode_->getFluidSolver().getVelocity().y;
        const double w0 = C / 3.0;
        const double w1 = C / 6.0;
        const double tauI = 1.0 / this->getTau();
        double temp[5];
        temp[T] = w0;
        temp[E] = w1 * (1.0 + ux * 3.0);
        temp[N] = w1 * (1.0 + uy * 3.0);
        temp[W] = w1 * (1.0 + (-ux) * 3.0);
        temp[S] = w1 * (1.0 + (-uy) * 3.0);
        const double R = reaction(C);
        const double deltaT = 1.0;
        const double r0 = deltaT * R / 3.0;
        const double r1 = deltaT * R / 6.0;
        d_[T] = d_[T] - d_[T] * tauI + temp[T] * tauI + r0;
        d_[E] = d_[E] - d_[E] * tauI + temp[E] * tauI + r1;
        d_[N] = d_[N] - d_[N] * tauI + temp[N] * tauI + r1;
        d_[W] = d_[W] - d_[W] * tauI + temp[W] * tauI + r1;
        d_[S] = d_[S] - d_[S] * tauI + temp[S] * tauI + r1;
        std::swap(d_[E], d_[W]);
        std::swap(d_[N], d_[S]);
    }

    virtual void advect() {
        std::swap(d_[getInverseDirection(W)],
                  this->physicalNode_->getPhysicalNeighbour(W)->getCDESolver(this->solverID_).accessDistribution(W));
        std::swap(d_[getInverseDirection(S)],
                  this->physicalNode_->getPhysicalNeighbour(S)->getCDESolver(this->solverID_).accessDistribution(S));
    }

    virtual double calculateEquilibrium(const Direction& dir) {
        const double C = getC();
        const double u = this->physicalNode_->getFluidSolver().getVelocity().x;
        const double v = this->physicalNode_->getFluidSolver().getVelocity().y;
        const double w1 = C / 6.0;
        switch (dir) {
            case T: return C / 3.0;
            case E: return w1 * (1.0 + u * 3.0);
            case N: return w1 * (1.0 + v * 3.0);
            case W: return w1 * (1.0 + (-u) * 3.0);
            case S: return w1 * (1.0 + (-v) * 3.0);
            default: return 0.0;
        }
    }

    virtual double& accessDistribution(const Direction& dir) { return d_[dir]; }

    virtual void rescaleDistributions(const double factor) {
        for (auto& it : d_) it *= factor;
    }

    virtual double getC() const { return std::accumulate(d_.begin(), d_.end(), 0.0); }

    // Same neighbour rule as CDESolverD2Q5::reinitialise (CDESolverD2Q5.cpp:156-228),
    // including its reads of getBoundaryNeighbour() for the diagonal directions.
    virtual void reinitialise() {
        double sumC = 0.0;
        int counter = 0;
        const unsigned int my = this->physicalNode_->getDomainIdentifier();
        std::array<Direction, 4> dir1{{E, N, W, S}};
        for (auto d : dir1) {
            if ((this->physicalNode_->getBoundaryNeighbour(d) == nullptr) &&
                (my == this->physicalNode_->getPhysicalNeighbour(d)->getDomainIdentifier())) {
                sumC += this->physicalNode_->getPhysicalNeighbour(d)->getCDESolver(this->solverID_).getC();
                counter++;
            }
        }
        if (counter == 0) {
            std::array<Direction, 4> dir2{{NE, NW, SW, SE}};
            for (auto d : dir2) {
                if ((this->physicalNode_->getBoundaryNeighbour(d) == nullptr) &&
                    (my == this->physicalNode_->getPhysicalNeighbour(d)->getDomainIdentifier())) {
                    sumC += this->physicalNode_->getPhysicalNeighbour(d)->getCDESolver(this->solverID_).getC();
                    counter++;
                }
            }
            if (counter != 0) lbibref::registry().diagonalReinit++;
        }
        if (counter == 0) lbibref::registry().failedReinit++;
        sumC /= static_cast<double>(counter);
        for (int d = 0; d < 5; ++d) d_[d] = sumC / 5.0;
        this->collide();
    }

    virtual void loadSolver(std::stringstream* const stream) {
        int x, y;
        (*stream) >> x >> y;
        for (int d = 0; d < 5; ++d) (*stream) >> d_[d];
    }

    virtual void writeSolver(std::ostream* const stream) {
        (*stream) << this->physicalNode_->getXPos() << '\t' << this->physicalNode_->getYPos();
        for (auto d : d_) (*stream) << '\t' << d;
        (*stream) << '\n';
    }

 protected:
    std::array<double, 5> d_;
};

class LbibCDESolverD2Q5_A : public LbibCDE<LbibCDESolverD2Q5_A> {
 public:
    LbibCDESolverD2Q5_A();
    static const std::string name;
};
const std::string LbibCDESolverD2Q5_A::name = "LbibCDESolverD2Q5_A";

class LbibCDESolverD2Q5_B : public LbibCDE<LbibCDESolverD2Q5_B> {
 public:
    LbibCDESolverD2Q5_B();
    static const std::string name;
};
const std::string LbibCDESolverD2Q5_B::name = "LbibCDESolverD2Q5_B";

class LbibCDESolverD2Q5_C : public LbibCDE<LbibCDESolverD2Q5_C> {
 public:
    LbibCDESolverD2Q5_C();
    static const std::string name;
};
const std::string LbibCDESolverD2Q5_C::name = "LbibCDESolverD2Q5_C";

// Out-of-line constructors: defining them instantiates the base-class
// constructors, whose `reg = reg` triggers the factory self-registration
// (the same mechanism as CDEAbstractSolver.hpp:141-176).
LbibCDESolverD2Q5_A::LbibCDESolverD2Q5_A() {}
LbibCDESolverD2Q5_B::LbibCDESolverD2Q5_B() {}
LbibCDESolverD2Q5_C::LbibCDESolverD2Q5_C() {}
LbibMembraneTension::LbibMembraneTension() : BioBaseSolver() {}
LbibAreaRegulator::LbibAreaRegulator() : BioBaseSolver() {}
LbibCellJunction::LbibCellJunction() : BioBaseSolver() {}
LbibCellDivision::LbibCellDivision() : BioBaseSolver() {}

}  // namespace solver
}  // namespace LbmLib
