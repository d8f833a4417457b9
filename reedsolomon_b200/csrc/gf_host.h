// gf_host.h -- host-side GF(2^8) algebra for the classic codec.
//
// The encoding matrix, its inversions and the inversion-tree cache stay on
// the host (matrix.go, inversion_tree.go, reedsolomon.go:232-413); only the
// matrix x shards contraction runs on the GPU.
#pragma once

#include <cstdint>
#include <memory>
#include <mutex>
#include <shared_mutex>
#include <vector>

namespace rsgpu {

// Field GF(2^8) with generating polynomial x^8+x^4+x^3+x^2+1 (galois.go:26).
struct Gf256 {
    uint8_t log[256];
    uint8_t exp[256];
    uint8_t mul[256][256];
    uint8_t inv[256];
    static const Gf256 &get();

  private:
    Gf256();
};

inline uint8_t gf_mul(uint8_t a, uint8_t b) { return Gf256::get().mul[a][b]; }
uint8_t gf_exp(uint8_t a, int n);   // galExp (galois.go:898-912)
uint8_t gf_one_over(uint8_t a);     // galOneOver (galois.go:887-894)

// Row-major byte matrix.
struct Matrix {
    int rows = 0, cols = 0;
    std::vector<uint8_t> v;
    Matrix() = default;
    Matrix(int r, int c) : rows(r), cols(c), v((size_t)r * c, 0) {}
    uint8_t &at(int r, int c) { return v[(size_t)r * cols + c]; }
    uint8_t at(int r, int c) const { return v[(size_t)r * cols + c]; }
    const uint8_t *row(int r) const { return v.data() + (size_t)r * cols; }
};

Matrix mat_multiply(const Matrix &a, const Matrix &b);        // matrix.go:103-117
int mat_invert(const Matrix &m, Matrix &out);                 // matrix.go:192-265; returns rs status
int build_encoding_matrix(int kind, int k, int total, Matrix &out);  // reedsolomon.go:232-413
Matrix xor_matrix(int k);                                     // reedsolomon.go:391-413

// Thread-safe cache of decode matrices keyed by the sorted list of invalid
// row indices, lazily filled (inversion_tree.go:16-164).
class InversionTree {
  public:
    InversionTree(int data_shards, int parity_shards);
    std::shared_ptr<const Matrix> get(const std::vector<int> &invalid) const;
    void insert(const std::vector<int> &invalid, std::shared_ptr<const Matrix> m);

  private:
    struct Node {
        std::shared_ptr<const Matrix> matrix;
        std::vector<std::unique_ptr<Node>> children;
    };
    int total_;
    Node root_;
    mutable std::shared_mutex mu_;
};

}  // namespace rsgpu
