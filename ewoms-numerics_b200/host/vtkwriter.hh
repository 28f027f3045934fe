// VTK output of the lens simulation: one XML UnstructuredGrid file (.vtu) per written time step
// plus a ParaView collection (.pvd) that lists them with their times, like the reference's
// VtkMultiWriter (io/vtkmultiwriter.hh:123-193, 480-515; file names <simName>-<5-digit index>.vtu
// and <simName>.pvd) with the cell fields of VtkMultiPhaseModule (io/vtkmultiphasemodule.hh:
// 318-337): pressure_<phase>, density_<phase>, saturation_<phase>, mobility_<phase>,
// relativePerm_<phase>, viscosity_<phase>, porosity, intrinsicPerm; phases "w" and "n".
//
// Structured grids only: cells are axis-aligned quadrilaterals (2D) or hexahedra (3D) on the
// uniform grid [0,lx] x [0,ly] (x [0,lz]); points are the grid vertices, x fastest. Data is ASCII,
// per cell (cell-centred discretization) or per vertex (vertex-centred, written as PointData like
// the reference's vertex-centred VTK output).
#ifndef EWG_HOST_VTKWRITER_HH
#define EWG_HOST_VTKWRITER_HH

#include <cstdint>
#include <cstdio>
#include <fstream>
#include <iomanip>
#include <sstream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../../include/ewg.h"

namespace ewg {

class VtkMultiWriter {
public:
    // a named cell field with `components` values per cell (natural cell order)
    struct Field {
        std::string name;
        int components;
        std::vector<double> values;
    };

    VtkMultiWriter(std::string outputDir, std::string simName)
        : dir_(outputDir.empty() ? std::string(".") : std::move(outputDir)), name_(std::move(simName)) {}

    // Writes <dir>/<simName>-<index>.vtu for the state at `time` and rewrites the collection.
    // Returns the file name written.
    // pointData: the fields hold one value (x components) per grid vertex instead of per cell
    std::string write(double time, const ewg_grid& g, const std::vector<Field>& fields, bool pointData = false) {
        std::ostringstream fn;
        fn << name_ << "-" << std::setw(5) << std::setfill('0') << index_ << ".vtu";
        const std::string file = fn.str();
        writeVtu(dir_ + "/" + file, g, fields, pointData);
        steps_.emplace_back(time, file);
        writePvd();
        ++index_;
        return file;
    }

    static void writeVtu(const std::string& path, const ewg_grid& g, const std::vector<Field>& fields,
                         bool pointData = false) {
        const int dim = g.dim;
        const int nx = g.nx, ny = g.ny, nz = dim == 3 ? g.nz : 1;
        const int64_t nCells = (int64_t)nx * ny * nz;
        const int px = nx + 1, py = ny + 1, pz = dim == 3 ? nz + 1 : 1;
        const int64_t nPoints = (int64_t)px * py * pz;
        const int64_t nValues = pointData ? (int64_t)(nx + 1) * (ny + 1) * (dim == 3 ? nz + 1 : 1) : nCells;
        for (const Field& f : fields)
            if ((int64_t)f.values.size() != nValues * f.components)
                throw std::runtime_error("vtk field '" + f.name + "' has the wrong length");
        std::ofstream o(path);
        if (!o) throw std::runtime_error("cannot open '" + path + "' for writing");
        o << std::setprecision(17);
        o << "<?xml version=\"1.0\"?>\n"
          << "<VTKFile type=\"UnstructuredGrid\" version=\"0.1\" byte_order=\"LittleEndian\">\n"
          << " <UnstructuredGrid>\n"
          << "  <Piece NumberOfPoints=\"" << nPoints << "\" NumberOfCells=\"" << nCells << "\">\n";
        o << (pointData ? "   <PointData>\n" : "   <CellData>\n");
        for (const Field& f : fields) {
            o << "    <DataArray type=\"Float64\" Name=\"" << f.name << "\" NumberOfComponents=\"" << f.components
              << "\" format=\"ascii\">\n";
            for (size_t k = 0; k < f.values.size(); ++k) o << f.values[k] << ((k + 1) % 8 ? " " : "\n");
            o << "\n    </DataArray>\n";
        }
        o << (pointData ? "   </PointData>\n" : "   </CellData>\n");
        o << "   <Points>\n    <DataArray type=\"Float64\" NumberOfComponents=\"3\" format=\"ascii\">\n";
        const double hx = g.lx / nx, hy = g.ly / ny, hz = dim == 3 ? g.lz / nz : 0.0;
        for (int k = 0; k < pz; ++k)
            for (int j = 0; j < py; ++j)
                for (int i = 0; i < px; ++i) o << i * hx << " " << j * hy << " " << k * hz << "\n";
        o << "    </DataArray>\n   </Points>\n";
        o << "   <Cells>\n    <DataArray type=\"Int64\" Name=\"connectivity\" format=\"ascii\">\n";
        auto pid = [&](int i, int j, int k) { return ((int64_t)k * py + j) * px + i; };
        for (int k = 0; k < nz; ++k)
            for (int j = 0; j < ny; ++j)
                for (int i = 0; i < nx; ++i) {
                    // VTK_QUAD / VTK_HEXAHEDRON vertex order (counter-clockwise bottom, then top)
                    o << pid(i, j, k) << " " << pid(i + 1, j, k) << " " << pid(i + 1, j + 1, k) << " "
                      << pid(i, j + 1, k);
                    if (dim == 3)
                        o << " " << pid(i, j, k + 1) << " " << pid(i + 1, j, k + 1) << " " << pid(i + 1, j + 1, k + 1)
                          << " " << pid(i, j + 1, k + 1);
                    o << "\n";
                }
        o << "    </DataArray>\n    <DataArray type=\"Int64\" Name=\"offsets\" format=\"ascii\">\n";
        const int nv = dim == 3 ? 8 : 4;
        for (int64_t c = 0; c < nCells; ++c) o << (c + 1) * nv << ((c + 1) % 16 ? " " : "\n");
        o << "\n    </DataArray>\n    <DataArray type=\"UInt8\" Name=\"types\" format=\"ascii\">\n";
        for (int64_t c = 0; c < nCells; ++c) o << (dim == 3 ? 12 : 9) << ((c + 1) % 32 ? " " : "\n");
        o << "\n    </DataArray>\n   </Cells>\n  </Piece>\n </UnstructuredGrid>\n</VTKFile>\n";
        if (!o) throw std::runtime_error("error writing '" + path + "'");
    }

    // ---- restart (VtkMultiWriter::serialize / deserialize, io/vtkmultiwriter.hh:409-476) -------

    // index of the next file, the collection's text, and where its next entry goes (before the
    // closing tags, where the reference's open collection stream stands)
    int writerNum() const { return index_; }
    std::string collection() const { return pvdText(); }
    int64_t collectionWritePos() const {
        const std::string t = pvdText();
        return (int64_t)(t.size() - std::string(kPvdTail).size());
    }

    // Restores the writer from a restart file: the file index and the collection's entries
    // (parsed back from its text), and rewrites the collection file.
    void restore(int writerNum, const std::string& collection) {
        index_ = writerNum;
        steps_.clear();
        std::istringstream in(collection);
        std::string line;
        while (std::getline(in, line)) {
            const std::string ts = "timestep=\"", fs = "file=\"";
            const size_t a = line.find(ts), b = line.find(fs);
            if (a == std::string::npos || b == std::string::npos) continue;
            const size_t ae = line.find('"', a + ts.size()), be = line.find('"', b + fs.size());
            steps_.emplace_back(std::stod(line.substr(a + ts.size(), ae - a - ts.size())),
                                line.substr(b + fs.size(), be - b - fs.size()));
        }
        writePvd();
    }

private:
    static constexpr const char* kPvdTail = " </Collection>\n</VTKFile>\n";

    std::string pvdText() const {
        std::ostringstream o;
        o << std::setprecision(16);
        o << "<?xml version=\"1.0\"?>\n<VTKFile type=\"Collection\" version=\"0.1\" byte_order=\"LittleEndian\">\n"
          << " <Collection>\n";
        for (const auto& s : steps_)
            o << "   <DataSet timestep=\"" << s.first << "\" group=\"\" part=\"0\" file=\"" << s.second << "\"/>\n";
        o << kPvdTail;
        return o.str();
    }

    void writePvd() const {
        const std::string path = dir_ + "/" + name_ + ".pvd";
        std::ofstream o(path);
        if (!o) throw std::runtime_error("cannot open '" + path + "' for writing");
        o << pvdText();
    }

    std::string dir_, name_;
    int index_ = 0;
    std::vector<std::pair<double, std::string>> steps_;
};

}  // namespace ewg

#endif
