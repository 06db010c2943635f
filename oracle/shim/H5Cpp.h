/* Throw-on-use stand-in for the HDF5 C++ API.
 *
 * HDF5 is not installed in this image.  The reference only touches HDF5 in
 * the PyFR mesh/restart readers and writers (src/geometry.cpp:2387-3010,
 * src/solver.cpp:4275-4838), none of which is on the residual path.  This
 * header exists so those translation units compile; any call that would
 * reach the file system throws.  Test infrastructure only. */
#ifndef ORACLE_SHIM_H5CPP_H
#define ORACLE_SHIM_H5CPP_H

#include <cstddef>
#include <stdexcept>
#include <string>

#define _H5_NO_NAMESPACE

typedef long long hid_t;
typedef unsigned long long hsize_t;

#define H5F_ACC_RDONLY 0u
#define H5F_ACC_TRUNC 2u
#define H5S_SCALAR 0
#define H5S_SELECT_SET 0
#define H5T_VARIABLE ((size_t)-1)
#define H5T_C_S1 0
#define HOFFSET(S, M) offsetof(S, M)

enum H5T_class_t { H5T_FLOAT = 1, H5T_COMPOUND = 6 };
enum H5G_obj_t { H5G_DATASET = 1 };

[[noreturn]] inline void oracle_h5_unavailable()
{
  throw std::runtime_error("HDF5 is not available in the oracle build (.pyfrm/.pyfrs I/O disabled)");
}

inline hid_t H5Tcopy(hid_t) { oracle_h5_unavailable(); }
inline int H5Tset_size(hid_t, size_t) { oracle_h5_unavailable(); }

struct DataType
{
  DataType() {}
  DataType(hid_t) {}
};

struct PredType : DataType
{
  static const PredType NATIVE_DOUBLE;
  static const PredType NATIVE_INT;
  static const PredType NATIVE_INT8;
  static const PredType NATIVE_SHORT;
};

struct StrType : DataType
{
  StrType() {}
  StrType(int, size_t) {}
  StrType(hid_t) {}
};

struct CompType : DataType
{
  explicit CompType(size_t) {}
  void insertMember(const std::string &, size_t, const DataType &) {}
};

struct DataSpace
{
  DataSpace() {}
  DataSpace(int) {}
  DataSpace(int, const hsize_t *) {}
  DataSpace(int, const hsize_t *, const hsize_t *) {}
  int getSimpleExtentNdims() const { oracle_h5_unavailable(); }
  int getSimpleExtentDims(hsize_t *, hsize_t * = nullptr) const { oracle_h5_unavailable(); }
  void selectHyperslab(int, const hsize_t *, const hsize_t *, const hsize_t * = nullptr,
                       const hsize_t * = nullptr) { oracle_h5_unavailable(); }
  void close() {}
};

struct Attribute
{
  template <class... A> void write(A...) { oracle_h5_unavailable(); }
  template <class... A> void read(A...) { oracle_h5_unavailable(); }
};

struct DataSet
{
  DataType getDataType() const { oracle_h5_unavailable(); }
  DataSpace getSpace() const { oracle_h5_unavailable(); }
  H5T_class_t getTypeClass() const { oracle_h5_unavailable(); }
  template <class... A> void read(A &&...) const { oracle_h5_unavailable(); }
  template <class... A> void write(A &&...) const { oracle_h5_unavailable(); }
  template <class... A> Attribute createAttribute(A...) { oracle_h5_unavailable(); }
  void close() {}
};

struct H5File
{
  H5File(const std::string &, unsigned) { oracle_h5_unavailable(); }
  hsize_t getNumObjs() const { oracle_h5_unavailable(); }
  H5G_obj_t getObjTypeByIdx(hsize_t) const { oracle_h5_unavailable(); }
  std::string getObjnameByIdx(hsize_t) const { oracle_h5_unavailable(); }
  DataSet openDataSet(const std::string &) const { oracle_h5_unavailable(); }
  template <class... A> DataSet createDataSet(A...) { oracle_h5_unavailable(); }
  void close() {}
};

struct FileIException
{
  void printErrorStack() const {}
};

#endif
