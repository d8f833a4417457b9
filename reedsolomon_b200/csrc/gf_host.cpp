// gf_host.cpp -- host-side GF(2^8) algebra (see gf_host.h).
#include "gf_host.h"

#include "../../include/rsgpu.h"

namespace rsgpu {

Gf256::Gf256() {
    // Powers of the generator 2 modulo 0x11D give exp; log is its inverse.
    // Index 255 repeats index 0 as in galois.go:66-71.
    unsigned x = 1;
    for (int i = 0; i < 255; i++) {
        exp[i] = (uint8_t)x;
        x = (x << 1) ^ ((x & 0x80) ? 0x11D : 0);
    }
    exp[255] = exp[0];
    log[0] = 0;
    for (int i = 0; i < 255; i++) log[exp[i]] = (uint8_t)i;
    for (int a = 0; a < 256; a++)
        for (int b = 0; b < 256; b++)
            mul[a][b] = (a && b) ? exp[(log[a] + log[b]) % 255] : 0;
    inv[0] = 0;
    for (int a = 1; a < 256; a++) inv[a] = exp[(255 - log[a]) % 255];
}

const Gf256 &Gf256::get() {
    static const Gf256 g;
    return g;
}

uint8_t gf_exp(uint8_t a, int n) {
    if (n == 0) return 1;
    if (a == 0) return 0;
    const Gf256 &g = Gf256::get();
    int l = (int)g.log[a] * n;
    l %= 255;
    return g.exp[l];
}

uint8_t gf_one_over(uint8_t a) {
    const Gf256 &g = Gf256::get();
    return g.exp[(uint8_t)(g.log[a] ^ 255)];
}

Matrix mat_multiply(const Matrix &a, const Matrix &b) {
    const Gf256 &g = Gf256::get();
    Matrix r(a.rows, b.cols);
    for (int i = 0; i < a.rows; i++)
        for (int j = 0; j < b.cols; j++) {
            uint8_t s = 0;
            for (int t = 0; t < a.cols; t++) s ^= g.mul[a.at(i, t)][b.at(t, j)];
            r.at(i, j) = s;
        }
    return r;
}

// Gauss-Jordan elimination on [m | I].  Pivot search and row scaling follow
// matrix.go:209-265, so singular inputs are reported exactly when the
// reference reports errSingular.
int mat_invert(const Matrix &m, Matrix &out) {
    if (m.rows != m.cols) return RS_ERR_NOT_SQUARE;
    const Gf256 &g = Gf256::get();
    const int n = m.rows, w = 2 * n;
    std::vector<uint8_t> a((size_t)n * w, 0);
    for (int r = 0; r < n; r++) {
        for (int c = 0; c < n; c++) a[(size_t)r * w + c] = m.at(r, c);
        a[(size_t)r * w + n + r] = 1;
    }
    auto row = [&](int r) { return a.data() + (size_t)r * w; };
    for (int r = 0; r < n; r++) {
        if (row(r)[r] == 0) {
            for (int b = r + 1; b < n; b++)
                if (row(b)[r] != 0) {
                    for (int c = 0; c < w; c++) std::swap(row(r)[c], row(b)[c]);
                    break;
                }
        }
        if (row(r)[r] == 0) return RS_ERR_SINGULAR;
        if (row(r)[r] != 1) {
            uint8_t s = gf_one_over(row(r)[r]);
            for (int c = 0; c < w; c++) row(r)[c] = g.mul[row(r)[c]][s];
        }
        for (int b = r + 1; b < n; b++) {
            uint8_t s = row(b)[r];
            if (s)
                for (int c = 0; c < w; c++) row(b)[c] ^= g.mul[s][row(r)[c]];
        }
    }
    for (int d = 0; d < n; d++)
        for (int above = 0; above < d; above++) {
            uint8_t s = row(above)[d];
            if (s)
                for (int c = 0; c < w; c++) row(above)[c] ^= g.mul[s][row(d)[c]];
        }
    out = Matrix(n, n);
    for (int r = 0; r < n; r++)
        for (int c = 0; c < n; c++) out.at(r, c) = row(r)[n + c];
    return RS_OK;
}

static Matrix vandermonde(int rows, int cols) {
    Matrix vm(rows, cols);
    for (int r = 0; r < rows; r++)
        for (int c = 0; c < cols; c++) vm.at(r, c) = gf_exp((uint8_t)r, c);
    return vm;
}

Matrix xor_matrix(int k) {
    Matrix m(k + 1, k);
    for (int r = 0; r < k; r++) m.at(r, r) = 1;
    for (int c = 0; c < k; c++) m.at(k, c) = 1;
    return m;
}

static int build_jerasure(int k, int total, Matrix &vm) {
    const Gf256 &g = Gf256::get();
    vm = vandermonde(total, k);
    vm.at(0, 0) = 1;
    for (int i = 1; i < k; i++) vm.at(0, i) = 0;
    for (int i = 0; i < k - 1; i++) vm.at(total - 1, i) = 0;
    vm.at(total - 1, k - 1) = 1;
    for (int i = 0; i < k; i++) {
        int r = i;
        while (r < total && vm.at(r, i) == 0) r++;
        if (r != i)
            for (int c = 0; c < k; c++) std::swap(vm.at(r, c), vm.at(i, c));
        if (vm.at(i, i) != 1) {
            uint8_t t = gf_one_over(vm.at(i, i));
            for (int j = 0; j < total; j++) vm.at(j, i) = g.mul[vm.at(j, i)][t];
        }
        for (int j = 0; j < k; j++) {
            uint8_t t = vm.at(i, j);
            if (j != i && t)
                for (int rr = 0; rr < total; rr++) vm.at(rr, j) ^= g.mul[t][vm.at(rr, i)];
        }
    }
    for (int j = 0; j < k; j++) {
        uint8_t t = vm.at(k, j);
        if (t != 1) {
            t = gf_one_over(t);
            for (int i = k; i < total; i++) vm.at(i, j) = g.mul[vm.at(i, j)][t];
        }
    }
    for (int i = k + 1; i < total; i++) {
        uint8_t t = vm.at(i, 0);
        if (t != 1) {
            t = gf_one_over(t);
            for (int j = 0; j < k; j++) vm.at(i, j) = g.mul[vm.at(i, j)][t];
        }
    }
    return RS_OK;
}

int build_encoding_matrix(int kind, int k, int total, Matrix &out) {
    if (k <= 0 || total < k) return RS_ERR_INV_SHARD_NUM;
    const Gf256 &g = Gf256::get();
    switch (kind) {
    case RS_MATRIX_DEFAULT: {
        // Vandermonde times the inverse of its top square: systematic, and
        // every k-row subset stays invertible (reedsolomon.go:232-256).
        Matrix vm = vandermonde(total, k);
        Matrix top(k, k);
        for (int r = 0; r < k; r++)
            for (int c = 0; c < k; c++) top.at(r, c) = vm.at(r, c);
        Matrix inv;
        int rc = mat_invert(top, inv);
        if (rc) return rc;
        out = mat_multiply(vm, inv);
        return RS_OK;
    }
    case RS_MATRIX_JERASURE:
        return build_jerasure(k, total, out);
    case RS_MATRIX_CAUCHY:
        out = Matrix(total, k);
        for (int r = 0; r < total; r++)
            for (int c = 0; c < k; c++) out.at(r, c) = r < k ? (r == c) : g.inv[(uint8_t)(r ^ c)];
        return RS_OK;
    case RS_MATRIX_PAR1:
        out = Matrix(total, k);
        for (int r = 0; r < total; r++)
            for (int c = 0; c < k; c++)
                out.at(r, c) = r < k ? (r == c) : gf_exp((uint8_t)(c + 1), r - k);
        return RS_OK;
    }
    return RS_ERR_INVALID_INPUT;
}

InversionTree::InversionTree(int data_shards, int parity_shards)
    : total_(data_shards + parity_shards) {
    auto id = std::make_shared<Matrix>(data_shards, data_shards);
    for (int i = 0; i < data_shards; i++) id->at(i, i) = 1;
    root_.matrix = id;
    root_.children.resize(total_);
}

// Child slots are indexed relative to the previous invalid index plus one,
// since keys are sorted (inversion_tree.go:93-124).
std::shared_ptr<const Matrix> InversionTree::get(const std::vector<int> &invalid) const {
    std::shared_lock<std::shared_mutex> lk(mu_);
    if (invalid.empty()) return root_.matrix;
    const Node *n = &root_;
    int parent = 0;
    for (int idx : invalid) {
        int slot = idx - parent;
        if (slot < 0 || slot >= (int)n->children.size() || !n->children[slot]) return nullptr;
        n = n->children[slot].get();
        parent = idx + 1;
    }
    return n->matrix;
}

void InversionTree::insert(const std::vector<int> &invalid, std::shared_ptr<const Matrix> m) {
    if (invalid.empty()) return;  // root already holds the identity (inversion_tree.go:71-73)
    std::unique_lock<std::shared_mutex> lk(mu_);
    Node *n = &root_;
    int parent = 0;
    for (int idx : invalid) {
        int slot = idx - parent;
        if (slot < 0 || slot >= (int)n->children.size()) return;
        if (!n->children[slot]) {
            n->children[slot].reset(new Node());
            n->children[slot]->children.resize(total_ - idx);
        }
        n = n->children[slot].get();
        parent = idx + 1;
    }
    n->matrix = std::move(m);
}

}  // namespace rsgpu
