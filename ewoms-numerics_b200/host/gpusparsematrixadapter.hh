// Ewoms::Linear::GpuSparseMatrixAdapter<MatrixBlock, HostMatrix>: the SparseMatrixAdapter of the
// GPU path, whose values stay on the device.
//
//   using Block = Dune::FieldMatrix<Scalar, 2, 2>;
//   SET_TYPE_PROP(LensProblemEcfvAd, SparseMatrixAdapter,
//                 Ewoms::Linear::GpuSparseMatrixAdapter<Block, Dune::BCRSMatrix<Block>>);
//
// It has the interface of IstlSparseMatrixAdapter (linear/istlsparsematrixadapter.hh:52-165):
// the (rows, columns) and (simulator) constructors, reserve, istlMatrix, rows, cols, clear,
// clearRow, block, setBlock, addToBlock, commit and finalize. GpuEcfvLinearizer binds it to its
// device context and marks it device-current after every linearization; the Newton method then
// hands it from linearizer.jacobian() to the backend's prepare / setMatrix
// (nonlinear/newtonmethod.hh:371-374, :408) without a byte crossing PCIe, and
// GpuBiCGStabBackend::setMatrix solves on the device copy.
//
// A host consumer still sees a correct matrix: the first host read or write of a block (or of
// istlMatrix()) after a linearization exports the device Jacobian once into a HostMatrix with the
// reserved pattern (Dune::BCRSMatrix<MatrixBlock> in an eWoms build), and a host write marks the
// host copy as the newer one, which the GPU backend's setMatrix uploads before it solves. Only the
// structured-grid pattern of the cell-centred stencil (each row: the cell and its face
// neighbours, columns sorted) exists on the device; reserve() checks that the caller's pattern is
// that one when the first export compares them.
//
// HostMatrix needs the part of the dune-istl BCRSMatrix interface that
// IstlSparseMatrixAdapter::reserve uses (construction with BuildMode random, setrowsize,
// endrowsizes, addindex, endindices, operator[] of rows and of blocks, row iterators with index(),
// assignment of a scalar), and MatrixBlock the FieldMatrix interface field_type and [i][j].
#ifndef EWOMS_GPU_SPARSE_MATRIX_ADAPTER_HH
#define EWOMS_GPU_SPARSE_MATRIX_ADAPTER_HH

#include <cstddef>
#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "ewg.hh"

namespace Ewoms {
namespace Linear {

template <class MatrixBlockType, class HostMatrixType>
class GpuSparseMatrixAdapter
{
public:
    using IstlMatrix = HostMatrixType;
    using MatrixBlock = MatrixBlockType;
    using Scalar = typename MatrixBlock::field_type;

    // where the current values are
    enum class Residence { DeviceOnly, InSync, HostNewer };

    GpuSparseMatrixAdapter(const size_t rows, const size_t columns) : rows_(rows), columns_(columns) {}

    template <class Simulator>
    GpuSparseMatrixAdapter(const Simulator& simulator)
        : GpuSparseMatrixAdapter(simulator.model().numTotalDof(), simulator.model().numTotalDof())
    {}

    // IstlSparseMatrixAdapter::reserve: records the caller's pattern; the host matrix with this
    // pattern is built by the first export.
    template <class Set>
    void reserve(const std::vector<Set>& sparsityPattern)
    {
        if (sparsityPattern.size() != rows_)
            throw std::invalid_argument("GpuSparseMatrixAdapter::reserve: pattern has the wrong number of rows");
        patternRowPtr_.assign(rows_ + 1, 0);
        patternCols_.clear();
        for (size_t r = 0; r < rows_; ++r) {
            for (auto c : sparsityPattern[r])
                patternCols_.push_back(static_cast<int32_t>(c));
            patternRowPtr_[r + 1] = static_cast<int32_t>(patternCols_.size());
        }
        host_.reset();
    }

    // ---- device binding (used by GpuEcfvLinearizer and GpuBiCGStabBackend) ----------------------

    void bindDevice(ewg::Context* ctx) { ctx_ = ctx; }
    ewg::Context* deviceContext() const { return ctx_; }
    // a linearization wrote new values on the device
    void markDeviceCurrent() { residence_ = Residence::DeviceOnly; }
    Residence residence() const { return residence_; }
    // number of device -> host exports and host -> device uploads so far
    uint64_t exports() const { return exports_; }
    uint64_t uploads() const { return uploads_; }

    // Called by the GPU backend's setMatrix: after a host consumer changed blocks, the device
    // copy is replaced by the host copy. Otherwise nothing moves.
    void uploadIfHostNewer()
    {
        if (residence_ != Residence::HostNewer)
            return;
        requireDevice_("upload");
        std::vector<int32_t> rowPtr(rows_ + 1, 0), colIdx;
        std::vector<double> blocks;
        colIdx.reserve(patternCols_.size());
        blocks.reserve(4 * patternCols_.size());
        for (auto row = host_->begin(); row != host_->end(); ++row) {
            for (auto col = row->begin(); col != row->end(); ++col) {
                colIdx.push_back(static_cast<int32_t>(col.index()));
                for (int e = 0; e < 2; ++e)
                    for (int p = 0; p < 2; ++p)
                        blocks.push_back(static_cast<double>((*col)[e][p]));
            }
            rowPtr[row.index() + 1] = static_cast<int32_t>(colIdx.size());
        }
        ctx_->setMatrixBcrs(rowPtr.data(), colIdx.data(), blocks.data());
        ++uploads_;
        residence_ = Residence::InSync;
    }

    // ---- IstlSparseMatrixAdapter interface ---------------------------------------------------

    // Non-const access may change blocks: the host copy becomes the newer one.
    IstlMatrix& istlMatrix()
    {
        syncToHost_();
        residence_ = Residence::HostNewer;
        return *host_;
    }
    const IstlMatrix& istlMatrix() const
    {
        syncToHost_();
        return *host_;
    }

    size_t rows() const { return rows_; }
    size_t cols() const { return columns_; }

    void clear()
    {
        syncToHost_();
        (*host_) = Scalar(0.0);
        residence_ = Residence::HostNewer;
    }

    // IstlSparseMatrixAdapter::clearRow (istlsparsematrixadapter.hh:122-139)
    void clearRow(const size_t row, const Scalar diag = 1.0)
    {
        syncToHost_();
        MatrixBlock diagBlock(Scalar(0));
        for (int i = 0; i < 2; ++i)
            diagBlock[i][i] = diag;
        auto& matRow = (*host_)[row];
        for (auto colIt = matRow.begin(); colIt != matRow.end(); ++colIt) {
            if (colIt.index() == row)
                *colIt = diagBlock;
            else
                *colIt = Scalar(0.0);
        }
        residence_ = Residence::HostNewer;
    }

    void block(const size_t rowIdx, const size_t colIdx, MatrixBlock& value) const
    {
        syncToHost_();
        value = (*host_)[rowIdx][colIdx];
    }

    void setBlock(const size_t rowIdx, const size_t colIdx, const MatrixBlock& value)
    {
        syncToHost_();
        (*host_)[rowIdx][colIdx] = value;
        residence_ = Residence::HostNewer;
    }

    void addToBlock(const size_t rowIdx, const size_t colIdx, const MatrixBlock& value)
    {
        syncToHost_();
        (*host_)[rowIdx][colIdx] += value;
        residence_ = Residence::HostNewer;
    }

    void commit() {}
    void finalize() {}

private:
    void requireDevice_(const char* what) const
    {
        if (!ctx_)
            throw std::logic_error(std::string("GpuSparseMatrixAdapter: ") + what +
                                   " before a GPU linearizer bound the matrix to its device context");
    }

    // Export the device Jacobian into the host copy once per linearization.
    void syncToHost_() const
    {
        if (residence_ != Residence::DeviceOnly)
            return;
        requireDevice_("host access");
        const size_t n = static_cast<size_t>(ctx_->numCells());
        const size_t nnzb = static_cast<size_t>(ctx_->numBlocks());
        if (n != rows_)
            throw std::logic_error("GpuSparseMatrixAdapter: device context and matrix differ in size");
        std::vector<int32_t> rowPtr(n + 1), colIdx(nnzb);
        std::vector<double> blocks(4 * nnzb);
        ctx_->getJacobianBcrs(rowPtr.data(), colIdx.data(), blocks.data());
        if (!host_) {
            if (patternRowPtr_.empty()) {
                // no reserve(): take the device pattern
                patternRowPtr_ = rowPtr;
                patternCols_ = colIdx;
            }
            if (patternRowPtr_ != rowPtr || patternCols_ != colIdx)
                throw std::logic_error("GpuSparseMatrixAdapter: the reserved sparsity pattern is not the "
                                       "cell-centred stencil pattern the device assembles");
            // IstlSparseMatrixAdapter::reserve (istlsparsematrixadapter.hh:72-97)
            host_.reset(new IstlMatrix(rows_, columns_, IstlMatrix::random));
            for (size_t r = 0; r < rows_; ++r)
                host_->setrowsize(r, static_cast<size_t>(rowPtr[r + 1] - rowPtr[r]));
            host_->endrowsizes();
            for (size_t r = 0; r < rows_; ++r)
                for (int32_t q = rowPtr[r]; q < rowPtr[r + 1]; ++q)
                    host_->addindex(r, static_cast<size_t>(colIdx[q]));
            host_->endindices();
        }
        // rows of the host matrix iterate their columns in ascending order, as the export does
        for (size_t r = 0; r < rows_; ++r) {
            auto& row = (*host_)[r];
            auto it = row.begin();
            for (int32_t q = rowPtr[r]; q < rowPtr[r + 1]; ++q, ++it) {
                MatrixBlock& b = *it;
                b[0][0] = static_cast<Scalar>(blocks[4 * q]);
                b[0][1] = static_cast<Scalar>(blocks[4 * q + 1]);
                b[1][0] = static_cast<Scalar>(blocks[4 * q + 2]);
                b[1][1] = static_cast<Scalar>(blocks[4 * q + 3]);
            }
        }
        ++exports_;
        residence_ = Residence::InSync;
    }

    size_t rows_, columns_;
    ewg::Context* ctx_ = nullptr;
    mutable std::vector<int32_t> patternRowPtr_, patternCols_;
    mutable std::unique_ptr<IstlMatrix> host_;
    mutable Residence residence_ = Residence::DeviceOnly;
    mutable uint64_t exports_ = 0;
    uint64_t uploads_ = 0;
};

// true for GpuSparseMatrixAdapter<...>: the GPU linearizer and backend keep such a matrix on the
// device; any other SparseMatrixAdapter (IstlSparseMatrixAdapter) is exported and uploaded
template <class T>
struct IsGpuSparseMatrixAdapter : std::false_type {};
template <class B, class H>
struct IsGpuSparseMatrixAdapter<GpuSparseMatrixAdapter<B, H>> : std::true_type {};

}} // namespace Linear, Ewoms

#endif
