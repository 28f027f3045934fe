// Restart files of the lens simulation in the reference's format (io/restart.hh:36-271), so a run
// can be checkpointed and resumed like Simulator::serialize / Simulator::run with RestartTime
// (utils/simulator.hh:669-688, :923-979).
//
// File <outputDir>/<simName>_time=<t>_rank=<rank>.ers (t and rank formatted by an ostream with its
// default precision), text written with precision 20:
//   eWoms restart file: gridName='blubb' numCPUs=<P> myRank=<r> numElements=<N> numEdges=<E>
//       numVertices=<V>                 (one line; magic cookie, checked on reading)
//   <empty line>                        (end of section)
//   Simulator
//   <episodeIdx> <episodeStartTime> <episodeLength> <startTime> <time> <timeStepIdx>
//   <empty line>
//   VTKMultiWriter                      (only with VTK output, FvBaseProblem::serialize)
//   <writer index>
//   <collection length>  <collection write position>
//   <the .pvd collection's bytes>
//   <empty line>
//   Entities: Codim 0                   (EcfvDiscretization::serialize, ecfvdiscretization.hh:186-188)
//   <p_w> <S_w>                         (one line per cell in the grid's natural order,
//   ...                                  FvBaseDiscretization::serializeEntity :1446-1460)
//   <empty line>
// Reading checks every section cookie and that no values are left in a section, throws on a
// missing file, an empty file or a short section (restart.hh:183-271), and sets solution(1) to
// the restored solution(0) (ecfvdiscretization.hh:197-201). The grid name is the reference's
// literal "blubb" (restart.hh:44), so files are exchangeable with its own.
#ifndef EWG_HOST_RESTART_HH
#define EWG_HOST_RESTART_HH

#include <cctype>
#include <cstdint>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../../include/ewg.h"

namespace ewg {

// Simulator's serialized state (utils/simulator.hh:944-952)
struct SimulatorState {
    int episodeIdx = 0;
    double episodeStartTime = 0.0;
    double episodeLength = 1e100;
    double startTime = 0.0;
    double time = 0.0;
    int timeStepIdx = 0;
};

class Restart {
public:
    // gridView.size(codim) of a structured grid: elements, entities of codim dim-1 (edges; the
    // faces of a 2D grid), vertices
    static void gridCounts(const ewg_grid& g, int64_t& elements, int64_t& edges, int64_t& vertices) {
        const int64_t nx = g.nx, ny = g.ny, nz = g.dim == 3 ? g.nz : 1;
        if (g.dim == 2) {
            elements = nx * ny;
            edges = nx * (ny + 1) + (nx + 1) * ny;
            vertices = (nx + 1) * (ny + 1);
        } else {
            elements = nx * ny * nz;
            edges = nx * (ny + 1) * (nz + 1) + (nx + 1) * ny * (nz + 1) + (nx + 1) * (ny + 1) * nz;
            vertices = (nx + 1) * (ny + 1) * (nz + 1);
        }
    }

    // magicRestartCookie_ (restart.hh:42-62)
    static std::string magicCookie(const ewg_grid& g, int numCPUs, int rank) {
        int64_t ne, ned, nv;
        gridCounts(g, ne, ned, nv);
        std::ostringstream oss;
        oss << "eWoms restart file: "
            << "gridName='blubb' "
            << "numCPUs=" << numCPUs << " "
            << "myRank=" << rank << " "
            << "numElements=" << ne << " "
            << "numEdges=" << ned << " "
            << "numVertices=" << nv;
        return oss.str();
    }

    // restartFileName_ (restart.hh:67-83)
    static std::string fileName(const std::string& outputDir, const std::string& simName, double t, int rank) {
        std::string dir = outputDir;
        if (dir == ".")
            dir = "";
        else if (!dir.empty() && dir.back() != '/')
            dir += "/";
        std::ostringstream oss;
        oss << dir << simName << "_time=" << t << "_rank=" << rank << ".ers";
        return oss.str();
    }

    const std::string& fileNameUsed() const { return fileName_; }

    // ---- writing -------------------------------------------------------------------------------

    void serializeBegin(const std::string& outputDir, const std::string& simName, double t, const ewg_grid& g,
                        int numCPUs = 1, int rank = 0) {
        fileName_ = fileName(outputDir, simName, t, rank);
        out_.open(fileName_.c_str());
        if (!out_.good()) throw std::runtime_error("Restart file '" + fileName_ + "' could not be created");
        out_.precision(20);
        serializeSectionBegin(magicCookie(g, numCPUs, rank));
        serializeSectionEnd();
    }
    std::ostream& serializeStream() { return out_; }
    void serializeSectionBegin(const std::string& cookie) { out_ << cookie << "\n"; }
    void serializeSectionEnd() { out_ << "\n"; }

    void serializeSimulator(const SimulatorState& s) {
        serializeSectionBegin("Simulator");
        out_ << s.episodeIdx << " " << s.episodeStartTime << " " << s.episodeLength << " " << s.startTime << " "
             << s.time << " " << s.timeStepIdx << " ";
        serializeSectionEnd();
    }

    // FvBaseProblem::serialize -> VtkMultiWriter::serialize (io/vtkmultiwriter.hh:409-437)
    void serializeVtkWriter(int writerNum, const std::string& collection, int64_t writePos) {
        serializeSectionBegin("VTKMultiWriter");
        out_ << writerNum << "\n";
        out_ << (int64_t)collection.size() << "  " << writePos << "\n";
        out_.write(collection.data(), (std::streamsize)collection.size());
        serializeSectionEnd();
    }

    // serializeEntities<0>: solution(0) of every cell, natural order, n x 2 values
    void serializeCells(const double* x, int64_t n) {
        serializeSectionBegin("Entities: Codim 0");
        for (int64_t c = 0; c < n; ++c) {
            if (!out_.good()) throw std::runtime_error("Could not serialize degree of freedom " + std::to_string(c));
            out_ << x[2 * c] << " " << x[2 * c + 1] << " " << "\n";
        }
        serializeSectionEnd();
    }

    void serializeEnd() {
        out_.close();
        if (out_.fail()) throw std::runtime_error("Restart file '" + fileName_ + "' could not be written");
    }

    // ---- reading -------------------------------------------------------------------------------

    void deserializeBegin(const std::string& outputDir, const std::string& simName, double t, const ewg_grid& g,
                          int numCPUs = 1, int rank = 0) {
        fileName_ = fileName(outputDir, simName, t, rank);
        in_.open(fileName_.c_str());
        if (!in_.good()) throw std::runtime_error("Restart file '" + fileName_ + "' could not be opened properly");
        in_.seekg(0, std::ios::end);
        if (in_.tellg() == 0) throw std::runtime_error("Restart file '" + fileName_ + "' is empty");
        in_.seekg(0, std::ios::beg);
        deserializeSectionBegin(magicCookie(g, numCPUs, rank));
        deserializeSectionEnd();
    }
    std::istream& deserializeStream() { return in_; }
    void deserializeSectionBegin(const std::string& cookie) {
        if (!in_.good()) throw std::runtime_error("Encountered unexpected EOF in restart file.");
        std::string buf;
        std::getline(in_, buf);
        if (buf != cookie) throw std::runtime_error("Could not start section '" + cookie + "'");
    }
    void deserializeSectionEnd() {
        std::string rest;
        std::getline(in_, rest);
        for (char ch : rest)
            if (!std::isspace((unsigned char)ch)) throw std::logic_error("Encountered unread values while deserializing");
    }

    void deserializeSimulator(SimulatorState& s) {
        deserializeSectionBegin("Simulator");
        in_ >> s.episodeIdx >> s.episodeStartTime >> s.episodeLength >> s.startTime >> s.time >> s.timeStepIdx;
        if (in_.fail()) throw std::runtime_error("Restart file is corrupted (Simulator section)");
        deserializeSectionEnd();
    }

    // VtkMultiWriter::deserialize (io/vtkmultiwriter.hh:443-476)
    void deserializeVtkWriter(int& writerNum, std::string& collection, int64_t& writePos) {
        deserializeSectionBegin("VTKMultiWriter");
        std::string dummy;
        in_ >> writerNum;
        std::getline(in_, dummy);
        int64_t len = 0;
        in_ >> len >> writePos;
        std::getline(in_, dummy);
        if (in_.fail() || len < 0) throw std::runtime_error("Restart file is corrupted (VTKMultiWriter section)");
        collection.assign((size_t)len, '\0');
        in_.read(&collection[0], (std::streamsize)len);
        if (in_.gcount() != (std::streamsize)len) throw std::runtime_error("Restart file is corrupted (VTK collection)");
        deserializeSectionEnd();
    }

    // deserializeEntities<0>: one line per cell with its two primary variables
    void deserializeCells(double* x, int64_t n) {
        deserializeSectionBegin("Entities: Codim 0");
        std::string line;
        for (int64_t c = 0; c < n; ++c) {
            if (!in_.good()) throw std::runtime_error("Restart file is corrupted");
            std::getline(in_, line);
            std::istringstream ls(line);
            for (int e = 0; e < 2; ++e) {
                if (!ls.good()) throw std::runtime_error("Could not deserialize degree of freedom " + std::to_string(c));
                ls >> x[2 * c + e];
                if (ls.fail()) throw std::runtime_error("Could not deserialize degree of freedom " + std::to_string(c));
            }
        }
        deserializeSectionEnd();
    }

    void deserializeEnd() { in_.close(); }

private:
    std::string fileName_;
    std::ifstream in_;
    std::ofstream out_;
};

}  // namespace ewg

#endif
