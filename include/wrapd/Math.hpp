/* Math.hpp -- the wrapd::math type names of the reference's src/Math.hpp:36-128
 * (Eigen aliases), for callers written against the reference.
 *
 * The headers in this directory (Math.hpp, Lame.hpp, ModelSettings.hpp,
 * Settings.hpp, RuntimeData.hpp, AlgorithmData.hpp, TetElements.hpp,
 * System.hpp, Solver.hpp) carry the reference's file names, class names and
 * public members, implemented over the C ABI of ../wrapd_gpu.h.  A program
 * written against the reference's src/ headers -- its samples/tests/quasi.cpp
 * with samples/utils/AddMeshes.hpp, for one -- builds against the GPU solver
 * by putting this directory on the include path in place of the reference's
 * src/ and linking libwrapd_gpu.so in place of the reference's sources.  The
 * caller supplies Eigen, as it does for the reference.  Only these type names
 * are kept; the reference's math routines (svd, polar, makePD) run inside the
 * library. */
#ifndef WRAPD_COMPAT_MATH_HPP
#define WRAPD_COMPAT_MATH_HPP

#include <Eigen/Dense>
#include <Eigen/Sparse>

#include <memory>
#include <string>
#include <vector>

namespace wrapd {
namespace math {

using VecX = Eigen::VectorXd;
using RowVecX = Eigen::RowVectorXd;
using VecXi = Eigen::VectorXi;
using MatX = Eigen::MatrixXd;
using MatXi = Eigen::MatrixXi;
using MatX2 = Eigen::MatrixX2d;
using Mat2X = Eigen::Matrix2Xd;
using MatX3 = Eigen::MatrixX3d;
using Mat3X = Eigen::Matrix3Xd;
using SpMat = Eigen::SparseMatrix<double, Eigen::RowMajor>;
using RowVec3 = Eigen::RowVector3d;
using RowVec4 = Eigen::RowVector4d;
using Triplet = Eigen::Triplet<double>;
using Triplets = std::vector<Triplet>;
using Doubles = std::vector<double>;
using AlignedBox = Eigen::AlignedBox<double, 3>;

template <int DIM> using Vec = Eigen::Matrix<double, DIM, 1>;
using Vec2 = Vec<2>;
using Vec3 = Vec<3>;
using Vec4 = Vec<4>;
template <int DIM> using Vecf = Eigen::Matrix<float, DIM, 1>;
using Vec2f = Vecf<2>;
using Vec3f = Vecf<3>;
template <int DIM> using Veci = Eigen::Matrix<int, DIM, 1>;
using Vec2i = Veci<2>;
using Vec3i = Veci<3>;
using Vec4i = Veci<4>;
template <int ROWS, int COLS> using Mat = Eigen::Matrix<double, ROWS, COLS>;
using Mat2x2 = Mat<2, 2>;
using Mat3x3 = Mat<3, 3>;
using Mat3x4 = Mat<3, 4>;
using Mat4x3 = Mat<4, 3>;
using Mat4x4 = Mat<4, 4>;

inline double clamp(double minval, double val, double maxval) {
    return val < minval ? minval : (val > maxval ? maxval : val);
}

/* Row-major n x 3 doubles <-> MatX3 (Eigen's default is column-major). */
inline std::vector<double> to_rows(const MatX3& X) {
    std::vector<double> v(3 * static_cast<size_t>(X.rows()));
    for (Eigen::Index i = 0; i < X.rows(); ++i)
        for (int c = 0; c < 3; ++c) v[3 * static_cast<size_t>(i) + c] = X(i, c);
    return v;
}
inline MatX3 from_rows(const double* v, Eigen::Index n) {
    MatX3 X(n, 3);
    for (Eigen::Index i = 0; i < n; ++i)
        for (int c = 0; c < 3; ++c) X(i, c) = v[3 * static_cast<size_t>(i) + c];
    return X;
}

}  // namespace math
}  // namespace wrapd

#endif  // WRAPD_COMPAT_MATH_HPP
