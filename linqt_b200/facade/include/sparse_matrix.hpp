// LinQT's sparse-operator interface (include/sparse_matrix.hpp of LinQT) on the B200
// library: the same class names and public members, implemented on the C ABI of
// include/linqt_gpu.h (linqt_b200/facade/facade.cpp).  The operator lives on the GPU as a
// linqt_op; the CSR arrays are kept on the host as the reference keeps them.
//
// Semantics kept from the reference: files and ConvertFromCSR hold the upper triangle of a
// Hermitian matrix (MKL HERMITIAN / UPPER descriptor, src/mkl_sparse_matrix.cpp:39-54);
// Multiply is y = a*H*x + b*y (:56-69); Rescale is H <- a*H + b*I (:73-97) and, as there,
// leaves rows()/cols()/vals() unchanged; BatchMultiply works on column-major blocks with
// leading dimension numRows() (:102-106).  MKL handles and descriptors are not exposed.
#ifndef SPARSE_MATRIX
#define SPARSE_MATRIX

#include <assert.h>

#include <complex>
#include <fstream>
#include <iostream>
#include <memory>
#include <string>
#include <vector>
using namespace std;  // the reference header exports std into its includers

struct linqt_op;

namespace Sparse {
// Reads LinQT's text CSR file (dim nnz / nnz "re im" / nnz columns / dim+1 row pointers).
bool OPERATOR_FromCSRFile(const std::string input, int &dim, vector<int> &columns, vector<int> &rowIndex,
                          vector<complex<double> > &values);
}  // namespace Sparse

class SparseMatrixType_BASE {
 public:
  typedef complex<double> value_t;
  typedef vector<value_t> vector_t;

  int numRows() { return numRows_; }
  int numCols() { return numCols_; }
  int rank() { return numRows() > numCols() ? numCols() : numRows(); }
  void setDimensions(const int numRows, const int numCols) {
    numRows_ = numRows;
    numCols_ = numCols;
  }
  void SetID(string id) { id_ = id; }
  string ID() const { return id_; }
  bool isIdentity() { return ID() == "1"; }

 private:
  int numRows_ = 0, numCols_ = 0;
  string id_;
};

class SparseMatrixType : public SparseMatrixType_BASE {
 public:
  SparseMatrixType() {}

  string matrixType() const { return "CSR Matrix on the GPU (linqt_b200)."; }
  void Multiply(const value_t a, const value_t *x, const value_t b, value_t *y);
  void Multiply(const value_t a, const vector_t &x, const value_t b, vector_t &y);
  void Rescale(const value_t a, const value_t b);
  void Multiply(const value_t *x, value_t *y) { Multiply(value_t(1, 0), x, value_t(0, 0), y); }
  void Multiply(const vector_t &x, vector_t &y) { Multiply(value_t(1, 0), x, value_t(0, 0), y); }
  void BatchMultiply(const int batchSize, const value_t a, const value_t *x, const value_t b, value_t *y);

  void ConvertFromCOO(vector<int> &rows, vector<int> &cols, vector<complex<double> > &vals);
  void ConvertFromCSR(vector<int> &rowIndex, vector<int> &cols, vector<complex<double> > &vals);

  vector<int> *rows() { return &rows_; }
  vector<int> *cols() { return &cols_; }
  vector<complex<double> > *vals() { return &vals_; }

  // the device operator (NULL before ConvertFromCSR / ConvertFromCOO)
  linqt_op *device_op() const { return op_.get(); }

 private:
  std::shared_ptr<linqt_op> op_;
  vector<int> rows_;
  vector<int> cols_;
  vector<complex<double> > vals_;
};

class SparseMatrixBuilder {
 public:
  void setSparseMatrix(SparseMatrixType *b) { _matrix_type = b; }
  void BuildOPFromCSRFile(const std::string input) {
    vector<int> columns, rowIndex;
    vector<complex<double> > values;
    int dim = 0;
    if (!Sparse::OPERATOR_FromCSRFile(input, dim, columns, rowIndex, values)) {
      std::cerr << "BuildOPFromCSRFile: cannot build an operator from " << input << std::endl;
      std::abort();
    }
    _matrix_type->setDimensions(dim, dim);
    _matrix_type->ConvertFromCSR(rowIndex, columns, values);
    std::cout << "OPERATOR SUCCESSFULLY BUILT" << std::endl;
  }
  SparseMatrixType *_matrix_type = nullptr;
};

#endif
