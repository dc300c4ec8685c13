// User-written models driven on the GPU through umc/device.cuh, as a user of
// the library would write them: three terms/models and two proposals with
// __host__ __device__ members, none of them known to libumc_b200.
//
//   CosineTerm   -- pair term E = -J cos(ti - tj), the XY model on angles as a
//                   PairModel (a user CellTerm of arity 2, term/cell.hpp:10-25);
//   PlaquetteTerm-- U(1) plaquette beta (1 - cos(t0 + t1 - t2 - t3)), arity 4,
//                   as a CellModel (term/plaquette.hpp:13-50);
//   DotTerm<N>   -- the Heisenberg pair term -J s_i . s_j, driven by Wolff
//                   (a PairModel is a WolffModel, driver.hpp:69-83);
//   IsingBondTerm + UpAxis -- the Ising pair term in int32 with FixedAxis,
//                   driven by Wolff;
//   WeightedIsing -- the reference graph test's IsingGraph: double spins and
//                   a coupling carried by every bond (PairGraph<double>),
//                   under Metropolis (FlipDouble) and Wolff (UnitAxis);
//   CubicHeisenberg -- a whole ModelLike (model.hpp:65-88) for the periodic
//                   cubic O(3) model whose neighbours come from the site index,
//                   with no bond table at all;
//   AngleShift   -- U1Shift (dof/u1.hpp:35-50): remainder(t + w (2u - 1), 2 pi);
//   Sphere3      -- UniformSphereN<3> (dof/vector.hpp:35-61);
//   SU2PlaquetteTerm + SU2Step -- a gauge group the library has no kernel for
//                   in this form: SU(2) links as unit quaternions (a user link
//                   type), the Wilson plaquette term and a symmetric left
//                   multiplication proposal.
//
// Exported with a C ABI for the Python tests and bench.py (ctypes): one-shot
// runs (um_xy_pair, um_xy_record, um_u1_cells, um_plaquette_u1, um_su2_2d,
// um_heisenberg_cubic, um_o3_wolff, um_ising_wolff, um_weighted_ising, um_lattice_o3) and persistent
// sessions (um_session_*) whose
// launches bench.py times.
#include <umc/device.cuh>

#include <cmath>
#include <cstdint>
#include <string>

namespace {

using namespace umc::gpu::device;

constexpr double kPi = 3.141592653589793238462643383279502884;

struct Angle
{
    using dtype = double;
    static constexpr std::size_t size = 1;
};

struct Spin
{
    using dtype = std::int8_t;
    static constexpr std::size_t size = 1;
};

// IsingTerm's arithmetic (term/ising.hpp:12-34): E = -J s_i s_j in int32.
struct IsingBondTerm
{
    using dtype = std::int8_t;
    using energy_type = std::int32_t;
    static constexpr std::size_t arity = 2;
    std::int32_t J;

    UMC_HD std::int32_t energy(const std::int8_t* const* l) const { return -J * (std::int32_t(*l[0]) * *l[1]); }
    UMC_HD std::int32_t delta(std::size_t which, const std::int8_t* old, const std::int8_t* nw,
                              const std::int8_t* const* l) const
    {
        const std::int8_t* fixed = l[which == 0 ? 1 : 0];
        return -J * (std::int32_t(*nw) * *fixed - std::int32_t(*old) * *fixed);
    }
};

// FixedAxis (dof/ising.hpp:41-49): the axis 1, no draw.
struct UpAxis
{
    template <class R>
    UMC_HD void sample(const std::int8_t*, R&, std::int8_t* out) const
    {
        out[0] = 1;
    }
};

// The weighted Ising model of the reference's graph test (test/graph_check.cpp:
// 34-83, IsingGraph): double spins, E = -sum over bonds of c s_i s_j with the
// coupling c carried by each bond of a PairGraph<double>.  A whole ModelLike
// and WolffModel over the weighted device rows (BondTables<double>::rows()):
// random-bond and weighted Ising models drop in this way.
struct WeightedIsing
{
    using value_type = double;
    static constexpr std::size_t size = 1;
    using bond_type = BondOf<double>;

    double* spin;
    PairRows<double> graph;

    UMC_HD std::size_t sites() const { return graph.sites(); }
    UMC_HD const double* data() const { return spin; }
    UMC_HD double* data() { return spin; }
    UMC_HD std::size_t degree(std::size_t i) const { return graph.degree(i); }
    UMC_HD const bond_type* bonds(std::size_t i) const { return graph.bonds(i); }
    UMC_HD std::uint32_t bond_id(std::size_t i, std::size_t a) const { return graph.bond_id(i, a); }

    UMC_HD double energy_at(std::size_t i) const
    {
        double e = 0.0;
        const bond_type* bs = graph.bonds(i);
        for (std::size_t a = 0; a < graph.degree(i); ++a) e += -bs[a].c * spin[i] * spin[bs[a].j];
        return e;
    }
    UMC_HD double energy_diff_at(std::size_t i, const double* p) const
    {
        double d = 0.0;
        const bond_type* bs = graph.bonds(i);
        for (std::size_t a = 0; a < graph.degree(i); ++a) d += -bs[a].c * (*p - spin[i]) * spin[bs[a].j];
        return d;
    }
    UMC_HD double energy_diff_bond(std::size_t i, const bond_type& b, const double* p) const
    {
        return -b.c * (*p - spin[b.j]) * spin[i];
    }
    UMC_HD void update(std::size_t i, const double* p) { spin[i] = *p; }
};

// The graph test's own Flip on double spins (test/graph_check.cpp:15-24) and
// its fixed reflection axis r = 1 (:27-32).
struct FlipDouble
{
    template <class R>
    UMC_HD void sample(const double* cur, R&, double* out) const
    {
        *out = *cur > 0.0 ? -1.0 : 1.0;
    }
    UMC_HD double log_ratio(const double*, const double*) const { return 0.0; }
};

struct UnitAxis
{
    template <class R>
    UMC_HD void sample(const double*, R&, double* out) const
    {
        out[0] = 1.0;
    }
};

template <std::size_t N>
struct Vec
{
    using dtype = double;
    static constexpr std::size_t size = N;
};

// E = -J s_i . s_j with HeisenbergTerm's arithmetic (term/heisenberg.hpp:11-35).
template <std::size_t N>
struct DotTerm
{
    using dtype = double;
    using energy_type = double;
    static constexpr std::size_t arity = 2;
    double J;

    UMC_HD static double dot(const double* a, const double* b)
    {
        double s = 0.0;
        for (std::size_t k = 0; k < N; ++k) s += a[k] * b[k];
        return s;
    }
    UMC_HD double energy(const double* const* l) const { return -J * dot(l[0], l[1]); }
    UMC_HD double delta(std::size_t which, const double* old, const double* nw, const double* const* l) const
    {
        const double* fixed = l[which == 0 ? 1 : 0];
        return -J * (dot(nw, fixed) - dot(old, fixed));
    }
};

struct CosineTerm
{
    using dtype = double;
    using energy_type = double;
    static constexpr std::size_t arity = 2;
    double J;

    UMC_HD double energy(const double* const* l) const { return -J * cos(*l[0] - *l[1]); }
    UMC_HD double delta(std::size_t which, const double* old, const double* nw, const double* const* l) const
    {
        const double fixed = *l[which == 0 ? 1 : 0];
        return -J * (cos(*nw - fixed) - cos(*old - fixed));
    }
};

struct PlaquetteTerm
{
    using dtype = double;
    using energy_type = double;
    static constexpr std::size_t arity = 4;
    double beta;

    UMC_HD static double plaq(const double* t) { return cos(t[0] + t[1] - t[2] - t[3]); }
    UMC_HD double energy(const double* const* l) const
    {
        const double t[4] = {*l[0], *l[1], *l[2], *l[3]};
        return beta * (1.0 - plaq(t));
    }
    UMC_HD double delta(std::size_t which, const double*, const double* nw, const double* const* l) const
    {
        double t[4] = {*l[0], *l[1], *l[2], *l[3]};
        const double before = plaq(t);
        t[which] = *nw;
        return beta * (before - plaq(t));
    }
};

// SU(2) links as unit quaternions: U = a0 + i (a1 s1 + a2 s2 + a3 s3), s_k
// the Pauli matrices, so (1/2) Tr U = a0, U^dagger = (a0, -a), and
// U V = (a0 b0 - a.b, a0 b + b0 a - a x b).
struct Quat
{
    double a[4];
};
struct SU2Dof
{
    using dtype = Quat;
    static constexpr std::size_t size = 1;
};
UMC_HD Quat qmul(const Quat& x, const Quat& y)
{
    const double* a = x.a;
    const double* b = y.a;
    return Quat{{a[0] * b[0] - a[1] * b[1] - a[2] * b[2] - a[3] * b[3],
                 a[0] * b[1] + b[0] * a[1] - (a[2] * b[3] - a[3] * b[2]),
                 a[0] * b[2] + b[0] * a[2] - (a[3] * b[1] - a[1] * b[3]),
                 a[0] * b[3] + b[0] * a[3] - (a[1] * b[2] - a[2] * b[1])}};
}
UMC_HD Quat qdag(const Quat& x) { return Quat{{x.a[0], -x.a[1], -x.a[2], -x.a[3]}}; }

// Wilson plaquette term beta (1 - (1/2) Tr U0 U1 U2^dagger U3^dagger) for SU(2),
// a user cell term of arity 4 with a user link type.
struct SU2PlaquetteTerm
{
    using dtype = Quat;
    using energy_type = double;
    static constexpr std::size_t arity = 4;
    double beta;

    UMC_HD static double half_trace(const Quat& u0, const Quat& u1, const Quat& u2, const Quat& u3)
    {
        return qmul(qmul(u0, u1), qmul(qdag(u3), qdag(u2))).a[0];  // U0 U1 (U3 U2)^dagger
    }
    UMC_HD double energy(const Quat* const* l) const { return beta * (1.0 - half_trace(*l[0], *l[1], *l[2], *l[3])); }
    UMC_HD double delta(std::size_t which, const Quat*, const Quat* nw, const Quat* const* l) const
    {
        Quat u[4] = {*l[0], *l[1], *l[2], *l[3]};
        const double before = half_trace(u[0], u[1], u[2], u[3]);
        u[which] = *nw;
        return beta * (before - half_trace(u[0], u[1], u[2], u[3]));
    }
};

// U -> R U with R = (cos t, sin t n), t uniform in [-w, w], n uniform on the
// sphere: R and R^dagger are equally likely, so the proposal is symmetric.
struct SU2Step
{
    double width;

    template <class R>
    UMC_HD void sample(const Quat* cur, R& rng, Quat* out) const
    {
        const double t = width * (2.0 * rng.uni() - 1.0);
        const double z = 2.0 * rng.uni() - 1.0;
        const double rr = sqrt(fmax(0.0, 1.0 - z * z));
        const double phi = 2.0 * kPi * rng.uni();
        const double st = sin(t);
        const Quat rot{{cos(t), st * rr * cos(phi), st * rr * sin(phi), st * z}};
        Quat u = qmul(rot, *cur);
        const double inv = 1.0 / sqrt(u.a[0] * u.a[0] + u.a[1] * u.a[1] + u.a[2] * u.a[2] + u.a[3] * u.a[3]);
        for (double& c : u.a) c *= inv;  // keep |U| = 1 against rounding drift
        *out = u;
    }
    UMC_HD double log_ratio(const Quat*, const Quat*) const { return 0.0; }
};

struct AngleShift
{
    double width;

    template <class R>
    UMC_HD void sample(const double* cur, R& rng, double* out) const
    {
        const double shift = width * (2.0 * rng.uni() - 1.0);
        out[0] = remainder(cur[0] + shift, 2.0 * kPi);
    }
    UMC_HD double log_ratio(const double*, const double*) const { return 0.0; }
};

struct Sphere3
{
    template <class R>
    UMC_HD void sample(const double*, R& rng, double* out) const
    {
        const double z = 2.0 * rng.uni() - 1.0;
        const double r = sqrt(1.0 - z * z);
        const double phi = 2.0 * kPi * rng.uni();
        out[0] = cos(phi) * r;
        out[1] = sin(phi) * r;
        out[2] = z;
    }
    UMC_HD double log_ratio(const double*, const double*) const { return 0.0; }
};

// Periodic Lx x Ly x Lz O(3) model, E = -J sum_<ij> S_i . S_j, site
// (z Ly + y) Lx + x; bonds to +-x, +-y, +-z computed from the index.
struct CubicHeisenberg
{
    using value_type = double;
    static constexpr std::size_t size = 3;
    double* s;
    std::uint32_t Lx, Ly, Lz;
    double J;

    UMC_HD std::size_t sites() const { return std::size_t(Lx) * Ly * Lz; }
    UMC_HD const double* data() const { return s; }
    UMC_HD double* data() { return s; }
    UMC_HD static double dot(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

    UMC_HD double energy_diff_at(std::size_t i, const double* p) const
    {
        const std::uint32_t x = std::uint32_t(i % Lx), y = std::uint32_t((i / Lx) % Ly),
                            z = std::uint32_t(i / (std::size_t(Lx) * Ly));
        const std::size_t nb[6] = {site((x + 1) % Lx, y, z), site((x + Lx - 1) % Lx, y, z),
                                   site(x, (y + 1) % Ly, z), site(x, (y + Ly - 1) % Ly, z),
                                   site(x, y, (z + 1) % Lz), site(x, y, (z + Lz - 1) % Lz)};
        const double* cur = s + i * 3;
        double d = 0.0;
        for (int a = 0; a < 6; ++a) d += -J * (dot(p, s + nb[a] * 3) - dot(cur, s + nb[a] * 3));
        return d;
    }
    UMC_HD double energy_at(std::size_t i) const
    {
        const std::uint32_t x = std::uint32_t(i % Lx), y = std::uint32_t((i / Lx) % Ly),
                            z = std::uint32_t(i / (std::size_t(Lx) * Ly));
        const double* cur = s + i * 3;
        return -J * (dot(cur, s + site((x + 1) % Lx, y, z) * 3) + dot(cur, s + site(x, (y + 1) % Ly, z) * 3) +
                     dot(cur, s + site(x, y, (z + 1) % Lz) * 3));
    }
    UMC_HD void update(std::size_t i, const double* p)
    {
        for (int k = 0; k < 3; ++k) s[i * 3 + k] = p[k];
    }
    UMC_HD std::size_t site(std::uint32_t x, std::uint32_t y, std::uint32_t z) const
    {
        return (std::size_t(z) * Ly + y) * Lx + x;
    }
};

// The same O(3) model written on the Model base (model.hpp:47-61), whose size
// is fixed at compile time: 8 x 8 x 8 sites.  The base holds the field and
// its write-back; the energy terms are CubicHeisenberg's on that field.
struct Heisenberg8 : Model<double, 512, 3>
{
    using value_type = double;
    static constexpr std::size_t size = 3;
    double J = 1.0;

    Heisenberg8(Field<double, 1536>& f, double J_) : Model(f), J(J_) {}
    // CubicHeisenberg only reads through its pointer in these two members
    UMC_HD CubicHeisenberg terms() const { return {const_cast<double*>(data()), 8, 8, 8, J}; }
    UMC_HD double energy_diff_at(std::size_t i, const double* p) const { return terms().energy_diff_at(i, p); }
    UMC_HD double energy_at(std::size_t i) const { return terms().energy_at(i); }
};

static_assert(ModelLike<CubicHeisenberg> && EnergyModel<CubicHeisenberg>);
static_assert(ModelLike<Heisenberg8> && EnergyModel<Heisenberg8>);
static_assert(WolffModel<PairModel<Vec<3>, DotTerm<3>>> && WolffModel<PairModel<Spin, IsingBondTerm>>);
static_assert(Axis<UpAxis, std::int8_t> && Axis<Sphere3, double>);
static_assert(WolffModel<LatticePairModel<Vec<3>, DotTerm<3>>> && EnergyModel<LatticePairModel<Vec<3>, DotTerm<3>>>);
static_assert(ModelLike<LatticeCellModel<Angle, PlaquetteTerm>> && CellEnergyModel<LatticeCellModel<Angle, PlaquetteTerm>>);
static_assert(CellTerm<SU2PlaquetteTerm, SU2Dof> && Proposal<SU2Step, Quat>);
static_assert(CellTerm<CosineTerm, Angle> && CellTerm<PlaquetteTerm, Angle>);
static_assert(Proposal<AngleShift, double> && Proposal<Sphere3, double>);

thread_local std::string g_error;

template <class F>
int guarded(F&& f)
{
    try {
        f();
        return 0;
    } catch (const std::exception& e) {
        g_error = e.what();
        return -1;
    }
}

}  // namespace

extern "C" {

const char* um_last_error(void) { return g_error.c_str(); }

// 1 when device.cuh's grid barrier gives up on a block that never arrives.
int um_barrier_selftest(int* timed_out)
{
    return guarded([&] { *timed_out = barrier_timeout_selftest() ? 1 : 0; });
}

// XY PairModel on a library pair graph: n_sweeps through sample(), recording
// energy_at_sum / 2 after every sweep; theta (sites) in/out.
int um_xy_pair(const umc_graph* g, double J, double beta, double width, std::uint64_t seed, std::uint64_t sweep0,
               std::uint32_t n_sweeps, double* theta, double* energies, std::uint32_t* grid)
{
    return guarded([&] {
        PairTables t(g);
        Buffer<double> field(t.sites());
        t.upload(field, theta, 1);
        auto model = t.model<Angle>(field.data(), CosineTerm{J});
        Metropolis<decltype(model), AngleShift> mc(model, AngleShift{width}, t.classes(), seed, beta);
        mc.set_sweeps(sweep0);
        std::uint32_t k = 0;
        mc.sample(n_sweeps, [&](const auto& m) { energies[k++] = 0.5 * m.energy_at_sum(); });
        t.download(field, theta, 1);
        if (grid) *grid = mc.grid();
    });
}

// XY as um_xy_pair, but the energies come from one launch that observes on
// the device (Metropolis::record_energy; energy_at summed, so 2E per sweep).
int um_xy_record(const umc_graph* g, double J, double beta, double width, std::uint64_t seed, std::uint64_t sweep0,
                 std::uint32_t n_sweeps, double* theta, double* energies)
{
    return guarded([&] {
        PairTables t(g);
        Buffer<double> field(t.sites());
        t.upload(field, theta, 1);
        auto model = t.model<Angle>(field.data(), CosineTerm{J});
        Metropolis<decltype(model), AngleShift> mc(model, AngleShift{width}, t.classes(), seed, beta);
        mc.set_sweeps(sweep0);
        mc.record_energy(n_sweeps, energies);
        for (std::uint32_t k = 0; k < n_sweeps; ++k) energies[k] *= 0.5;
        t.download(field, theta, 1);
    });
}

// U(1) CellModel on a library cell complex, n_sweeps in one launch; the total
// energy sum_c beta (1 - P_c) afterwards.
int um_u1_cells(const umc_cells* cc, double model_beta, double beta, double width, std::uint64_t seed,
                std::uint64_t sweep0, std::uint32_t n_sweeps, double* theta, double* total_energy)
{
    return guarded([&] {
        CellTables t(cc);
        Buffer<double> field(t.sites());
        t.upload(field, theta, 1);
        auto model = t.model<Angle>(field.data(), PlaquetteTerm{model_beta});
        Metropolis<decltype(model), AngleShift> mc(model, AngleShift{width}, t.classes(), seed, beta);
        mc.set_sweeps(sweep0);
        mc.run(n_sweeps);
        *total_energy = mc.total_energy();
        t.download(field, theta, 1);
    });
}

// U(1) with the user's PlaquetteTerm on a table-free PlaquetteLattice (L even;
// dim 2 = square_plaquettes, 4 = hypercubic_plaquettes), n_sweeps in one
// launch; the total energy afterwards.
int um_plaquette_u1(std::uint32_t L, std::uint32_t dim, double model_beta, double beta, double width,
                    std::uint64_t seed, std::uint64_t sweep0, std::uint32_t n_sweeps, double* theta,
                    double* total_energy)
{
    return guarded([&] {
        PlaquetteTables t(L, dim);
        Buffer<double> field(t.sites());
        t.upload(field, theta, 1);
        auto model = t.model<Angle>(field.data(), PlaquetteTerm{model_beta});
        Metropolis<decltype(model), AngleShift> mc(model, AngleShift{width}, t.classes(), seed, beta);
        mc.set_sweeps(sweep0);
        mc.run(n_sweeps);
        *total_energy = mc.total_energy();
        t.download(field, theta, 1);
    });
}

// 2D SU(2) with the user's quaternion links on the table-free L x L
// plaquettes, cold start: `warmup` sweeps, then n_sweeps recorded in one
// launch; plaq[s] = the mean (1/2) Tr U_p after sweep s.
int um_su2_2d(std::uint32_t L, double beta, double width, std::uint64_t seed, std::uint32_t warmup,
              std::uint32_t n_sweeps, double* plaq)
{
    return guarded([&] {
        PlaquetteTables t(L, 2);
        Buffer<Quat> field(t.sites());
        const std::vector<Quat> cold(t.sites(), Quat{{1.0, 0.0, 0.0, 0.0}});
        t.upload(field, cold.data(), 1);
        auto model = t.model<SU2Dof>(field.data(), SU2PlaquetteTerm{beta});
        Metropolis<decltype(model), SU2Step> mc(model, SU2Step{width}, t.classes(), seed, 1.0);
        mc.run(warmup);
        mc.record_energy(n_sweeps, plaq);
        for (std::uint32_t k = 0; k < n_sweeps; ++k) plaq[k] = 1.0 - plaq[k] / (beta * double(t.cells()));
    });
}

// Table-free O(3) ModelLike on a periodic cubic lattice (even extents),
// checkerboard classes; spins (sites x 3) in/out.
int um_heisenberg_cubic(std::uint32_t Lx, std::uint32_t Ly, std::uint32_t Lz, double J, double beta,
                        std::uint64_t seed, std::uint64_t sweep0, std::uint32_t n_sweeps, double* spins,
                        double* energy)
{
    return guarded([&] {
        const std::size_t n = std::size_t(Lx) * Ly * Lz;
        std::vector<std::uint32_t> colour(n);
        for (std::size_t i = 0; i < n; ++i) colour[i] = std::uint32_t((i % Lx + (i / Lx) % Ly + i / (std::size_t(Lx) * Ly)) & 1u);
        ClassTable classes(Classes::from_colours(colour, 2));
        Buffer<double> field(n * 3);
        field.upload(spins);
        CubicHeisenberg model{field.data(), Lx, Ly, Lz, J};
        Metropolis<CubicHeisenberg, Sphere3> mc(model, Sphere3{}, classes, seed, beta);
        mc.set_sweeps(sweep0);
        mc.run(n_sweeps);
        *energy = mc.energy_at_sum();
        field.download(spins);
    });
}

// Heisenberg8 (the Model base) from the same state and keys: the chain of
// um_heisenberg_cubic(8, 8, 8, ...).
int um_heisenberg_cubic8_base(double J, double beta, std::uint64_t seed, std::uint64_t sweep0, std::uint32_t n_sweeps,
                              double* spins, double* energy)
{
    return guarded([&] {
        constexpr std::size_t n = 512;
        std::vector<std::uint32_t> colour(n);
        for (std::size_t i = 0; i < n; ++i) colour[i] = std::uint32_t((i % 8 + (i / 8) % 8 + i / 64) & 1u);
        ClassTable classes(Classes::from_colours(colour, 2));
        Field<double, 3 * n> field;
        field.upload(spins);
        Heisenberg8 model(field, J);
        Metropolis<Heisenberg8, Sphere3> mc(model, Sphere3{}, classes, seed, beta);
        mc.set_sweeps(sweep0);
        mc.run(n_sweeps);
        *energy = mc.energy_at_sum();
        field.download(spins);
    });
}

// O(3) Wolff on a library pair graph with the user's DotTerm<3> and Sphere3
// axis.  sweeps == 0: n flips, their sizes to `sizes`; sweeps == 1: n Wolff
// sweeps (flips until the flipped sites add up to the lattice).  spins
// (sites x 3, site order) in/out.
int um_o3_wolff(const umc_graph* g, double J, double beta, std::uint64_t seed, std::uint64_t flip0, std::uint32_t n,
                int sweeps, double* spins, std::uint64_t* sizes, std::uint64_t* flips_done, double* mean_size)
{
    return guarded([&] {
        PairTables t(g);
        Buffer<double> field(std::size_t(t.sites()) * 3);
        t.upload(field, spins, 3);
        auto model = t.model<Vec<3>>(field.data(), DotTerm<3>{J});
        Wolff<decltype(model), Sphere3> w(model, Sphere3{}, t, seed, beta);
        w.set_flips(flip0);
        if (sweeps)
            w.run(n);
        else
            w.flips(n, sizes);
        *flips_done = w.flips_done() - flip0;
        *mean_size = w.mean_cluster_size();
        t.download(field, spins, 3);
    });
}

// Ising Wolff (IsingBondTerm, UpAxis) on a library pair graph: n flips, their
// sizes to `sizes`; spins (sites, site order) in/out.  tiled: the driver gets
// the tables (shared-memory tile labelling) or not (global union-find only).
int um_ising_wolff(const umc_graph* g, std::int32_t J, double beta, std::uint64_t seed, std::uint64_t flip0,
                   std::uint32_t n, std::int8_t* spins, std::uint64_t* sizes, int tiled)
{
    return guarded([&] {
        PairTables t(g);
        Buffer<std::int8_t> field(t.sites());
        t.upload(field, spins, 1);
        auto model = t.model<Spin>(field.data(), IsingBondTerm{J});
        using W = Wolff<decltype(model), UpAxis>;
        W w = tiled ? W(model, UpAxis{}, t, seed, beta) : W(model, UpAxis{}, seed, beta);
        w.set_flips(flip0);
        w.flips(n, sizes);
        t.download(field, spins, 1);
    });
}

// The weighted Ising model (WeightedIsing, FlipDouble, UnitAxis) on a library
// pair graph built with a double payload per bond (the coupling): wolff == 0,
// n Metropolis sweeps from sweep `first`, energies[k] = E after sweep k (may be
// NULL); wolff == 1, n Wolff flips from flip `first`, their sizes to `sizes`
// and E after each to `energies` (either may be NULL).  tiled: the Wolff
// driver gets the tables (shared-memory tile labelling).  spins (sites, site
// order) in/out.
int um_weighted_ising(const umc_graph* g, double beta, std::uint64_t seed, std::uint64_t first, std::uint32_t n,
                      int wolff, int tiled, double* spins, double* energies, std::uint64_t* sizes)
{
    return guarded([&] {
        BondTables<double> t(g);
        Buffer<double> field(t.sites());
        t.upload(field, spins, 1);
        WeightedIsing model{field.data(), t.rows()};
        if (wolff) {
            using W = Wolff<WeightedIsing, UnitAxis>;
            W w = tiled ? W(model, UnitAxis{}, t, seed, beta) : W(model, UnitAxis{}, seed, beta);
            w.set_flips(first);
            for (std::uint32_t k = 0; k < n; ++k) {
                std::uint64_t sz = 0;
                w.flips(1, &sz);
                if (sizes) sizes[k] = sz;
                if (energies) energies[k] = 0.5 * w.energy_at_sum();
            }
        } else {
            Metropolis<WeightedIsing, FlipDouble> mc(model, FlipDouble{}, t.classes(), seed, beta);
            mc.set_sweeps(first);
            std::uint32_t k = 0;
            mc.sample(n, [&](const auto& m) {
                if (energies) energies[k] = 0.5 * m.energy_at_sum();
                ++k;
            });
        }
        t.download(field, spins, 1);
    });
}

// O(3) with the user's DotTerm<3> on a table-free RegularLattice (Lx even,
// Ly and Lz even or 1): wolff == 0, n Metropolis sweeps with Sphere3 from
// sweep `first`; wolff == 1, n Wolff flips with the Sphere3 axis from flip
// `first`, sizes to `sizes`.  spins (sites x 3, site order) in/out.
int um_lattice_o3(std::uint32_t Lx, std::uint32_t Ly, std::uint32_t Lz, double J, double beta, std::uint64_t seed,
                  std::uint64_t first, std::uint32_t n, int wolff, double* spins, std::uint64_t* sizes)
{
    return guarded([&] {
        LatticeTables t(RegularLattice{Lx, Ly, Lz});
        Buffer<double> field(std::size_t(t.sites()) * 3);
        t.upload(field, spins, 3);
        auto model = t.model<Vec<3>>(field.data(), DotTerm<3>{J});
        if (wolff) {
            Wolff<decltype(model), Sphere3> w(model, Sphere3{}, t, seed, beta);
            w.set_flips(first);
            w.flips(n, sizes);
        } else {
            Metropolis<decltype(model), Sphere3> mc(model, Sphere3{}, t.classes(), seed, beta);
            mc.set_sweeps(first);
            mc.run(n);
        }
        t.download(field, spins, 3);
    });
}

}  // extern "C"

// ---- persistent sessions: tables, field and driver stay on the device; the
// launches bench.py times.  Kinds:
//   0  XY (CosineTerm + AngleShift, FP64) on a library pair graph's tables;
//   1  O(3) (DotTerm<3, float> + SphereF, FP32) on a table-free RegularLattice;
//   2  the same O(3) model on the lattice's CSR tables (PairTables);
//   3  Ising Wolff (IsingBondTerm + UpAxis) on a library pair graph's tables;
//   4  U(1) (PlaquetteTerm + AngleShift, FP64) on hypercubic_plaquettes(L) tables;
//   5  the same on the table-free PlaquetteLattice(L, 4).
namespace {

template <class T, std::size_t N>
struct VecT
{
    using dtype = T;
    static constexpr std::size_t size = N;
};

// E = -J s_i . s_j in the spins' own precision.
template <class T, std::size_t N>
struct DotTermT
{
    using dtype = T;
    using energy_type = T;
    static constexpr std::size_t arity = 2;
    T J;

    UMC_HD static T dot(const T* a, const T* b)
    {
        T s = 0;
        for (std::size_t k = 0; k < N; ++k) s += a[k] * b[k];
        return s;
    }
    UMC_HD T energy(const T* const* l) const { return -J * dot(l[0], l[1]); }
    UMC_HD T delta(std::size_t which, const T* old, const T* nw, const T* const* l) const
    {
        const T* fixed = l[which == 0 ? 1 : 0];
        return -J * (dot(nw, fixed) - dot(old, fixed));
    }
};

// UniformSphereN<3> in FP32: height z = 2u - 1, angle 2 pi u.
struct SphereF
{
    template <class R>
    UMC_HD void sample(const float*, R& rng, float* out) const
    {
        const float z = float(2.0 * rng.uni() - 1.0);
        const float r = sqrtf(fmaxf(0.f, 1.f - z * z));
        float sn, cs;
        sincospif(float(2.0 * rng.uni()), &sn, &cs);
        out[0] = cs * r;
        out[1] = sn * r;
        out[2] = z;
    }
    UMC_HD float log_ratio(const float*, const float*) const { return 0.f; }
};

struct SessionBase
{
    static cudaStream_t make_stream()
    {
        cudaStream_t s = nullptr;
        cuda_check(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "stream");
        return s;
    }
    SessionBase() : stream(make_stream()) {}
    virtual ~SessionBase()
    {
        for (auto& e : pending) {
            cudaEventDestroy(e.first);
            cudaEventDestroy(e.second);
        }
        cudaStreamDestroy(stream);
    }
    virtual void set_field(const void* host) = 0;
    virtual void get_field(void* host) = 0;
    virtual void launch(std::uint64_t sweeps) = 0;
    virtual void check() = 0;
    virtual double energy() = 0;
    virtual std::uint64_t sweeps() const = 0;
    virtual std::uint32_t grid() const = 0;
    // Sites each step updated since the last call (Wolff: cluster sizes).
    virtual std::vector<std::uint64_t> take_sizes() { return {}; }

    void fold()
    {
        cuda_check(cudaStreamSynchronize(stream), "sync");
        for (auto& e : pending) {
            float ms = 0.f;
            cuda_check(cudaEventElapsedTime(&ms, e.first, e.second), "event");
            timed_ms += ms;
            cudaEventDestroy(e.first);
            cudaEventDestroy(e.second);
        }
        pending.clear();
    }

    cudaStream_t stream;
    bool timing = false;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pending;
    std::uint64_t launches = 0;
    double timed_ms = 0.0;
};

// Tables + field + Metropolis; `scalars` field values per site.
template <class Tables, class D, class Term, class Q>
struct Session final : SessionBase
{
    using T = typename D::dtype;
    template <class Src>
    Session(const Src& src, Term term, Q q, double beta, std::uint64_t seed)
        : tables(src), field(std::size_t(tables.sites()) * D::size),
          mc(tables.template model<D>(field.data(), term), q, tables.classes(), seed, beta, stream)
    {}
    void set_field(const void* host) override { tables.upload(field, static_cast<const T*>(host), D::size, stream); }
    void get_field(void* host) override { tables.download(field, static_cast<T*>(host), D::size, stream); }
    void launch(std::uint64_t sweeps) override { mc.enqueue(sweeps); }
    void check() override { mc.check(); }
    double energy() override
    {
        if constexpr (requires { mc.total_energy(); })
            return mc.total_energy();  // a cell model: the sum over cells
        else
            return 0.5 * mc.energy_at_sum();  // a pair model: every bond at both ends
    }
    std::uint64_t sweeps() const override { return mc.sweeps(); }
    std::uint32_t grid() const override { return mc.grid(); }

    Tables tables;
    Buffer<T> field;
    Metropolis<decltype(std::declval<Tables&>().template model<D>(nullptr, std::declval<Term>())), Q> mc;
};

// Ising Wolff (IsingBondTerm + UpAxis) on a library pair graph's tables; a
// launch is n flips, and their sizes are kept for take_sizes().
struct IsingWolffSession final : SessionBase
{
    IsingWolffSession(const umc_graph* g, std::int32_t J, double beta, std::uint64_t seed)
        : tables(g), field(tables.sites()),
          w(tables.model<Spin>(field.data(), IsingBondTerm{J}), UpAxis{}, tables, seed, beta, stream)
    {}
    void set_field(const void* host) override { tables.upload(field, static_cast<const std::int8_t*>(host), 1, stream); }
    void get_field(void* host) override { tables.download(field, static_cast<std::int8_t*>(host), 1, stream); }
    void launch(std::uint64_t n) override
    {
        const std::size_t at = sizes.size();
        sizes.resize(at + n);
        w.flips(n, sizes.data() + at);
    }
    void check() override {}
    double energy() override { return 0.5 * w.energy_at_sum(); }
    std::uint64_t sweeps() const override { return w.flips_done(); }
    std::uint32_t grid() const override { return w.grid(); }
    std::vector<std::uint64_t> take_sizes() override { return std::exchange(sizes, {}); }

    PairTables tables;
    Buffer<std::int8_t> field;
    Wolff<PairModel<Spin, IsingBondTerm>, UpAxis> w;
    std::vector<std::uint64_t> sizes;
};

using XYSession = Session<PairTables, Angle, CosineTerm, AngleShift>;
using U1CellSession = Session<CellTables, Angle, PlaquetteTerm, AngleShift>;
using U1PlaquetteSession = Session<PlaquetteTables, Angle, PlaquetteTerm, AngleShift>;
using O3LatticeSession = Session<LatticeTables, VecT<float, 3>, DotTermT<float, 3>, SphereF>;
using O3TableSession = Session<PairTables, VecT<float, 3>, DotTermT<float, 3>, SphereF>;

// The lattice's own CSR as a library graph, for the table variant.
struct LatticeGraph
{
    umc_graph* g = nullptr;
    LatticeGraph(std::uint32_t Lx, std::uint32_t Ly, std::uint32_t Lz)
    {
        umc_check(Lz > 1 ? umc_graph_cubic(Lx, Ly, Lz, &g) : umc_graph_square(Lx, Ly, &g));
    }
    ~LatticeGraph() { umc_graph_destroy(g); }
};

}  // namespace

extern "C" {

// kind 0: graph, J, beta, width (dims unused); kinds 1, 2: dims Lx, Ly, Lz, J,
// beta; kind 3: graph, J (an integer), beta.
int um_session_create(int kind, const umc_graph* g, std::uint32_t Lx, std::uint32_t Ly, std::uint32_t Lz, double J,
                      double beta, double width, std::uint64_t seed, void** out)
{
    return guarded([&] {
        if (kind == 0) {
            *out = static_cast<SessionBase*>(new XYSession(g, CosineTerm{J}, AngleShift{width}, beta, seed));
        } else if (kind == 1) {
            *out = static_cast<SessionBase*>(
                new O3LatticeSession(RegularLattice{Lx, Ly, Lz}, DotTermT<float, 3>{float(J)}, SphereF{}, beta, seed));
        } else if (kind == 2) {
            LatticeGraph lg(Lx, Ly, Lz);
            *out = static_cast<SessionBase*>(
                new O3TableSession(lg.g, DotTermT<float, 3>{float(J)}, SphereF{}, beta, seed));
        } else if (kind == 3) {
            *out = static_cast<SessionBase*>(new IsingWolffSession(g, std::int32_t(J), beta, seed));
        } else if (kind == 4 || kind == 5) {
            // U(1) plaquettes on L^4 (Lx = L): J is the model's beta, width the shift
            umc_cells* cc = nullptr;
            umc_check(umc_cells_hypercubic(Lx, &cc));
            struct Free
            {
                umc_cells* c;
                ~Free() { umc_cells_destroy(c); }
            } guard{cc};
            if (kind == 4)
                *out = static_cast<SessionBase*>(new U1CellSession(cc, PlaquetteTerm{J}, AngleShift{width}, beta, seed));
            else
                *out = static_cast<SessionBase*>(
                    new U1PlaquetteSession(PlaquetteLattice(Lx, 4), PlaquetteTerm{J}, AngleShift{width}, beta, seed));
        } else {
            throw std::invalid_argument("unknown session kind");
        }
    });
}

void um_session_destroy(void* h) { delete static_cast<SessionBase*>(h); }

void* um_session_stream(void* h) { return static_cast<SessionBase*>(h)->stream; }

// Field from/to host memory (site order, the model's dtype), ordered on the
// session's stream; set_field returns before the copy completes.
int um_session_set_field(void* h, const void* host)
{
    return guarded([&] { static_cast<SessionBase*>(h)->set_field(host); });
}
int um_session_get_field(void* h, void* host)
{
    return guarded([&] { static_cast<SessionBase*>(h)->get_field(host); });
}

// n sweeps in one launch, not waited for; with timing on, CUDA events bracket it.
int um_session_enqueue(void* h, std::uint64_t sweeps)
{
    return guarded([&] {
        auto* s = static_cast<SessionBase*>(h);
        cudaEvent_t a = nullptr, b = nullptr;
        if (s->timing) {
            cuda_check(cudaEventCreate(&a), "event");
            cuda_check(cudaEventCreate(&b), "event");
            cuda_check(cudaEventRecord(a, s->stream), "event");
        }
        s->launch(sweeps);
        s->launches += (sweeps + (1u << 30) - 1) >> 30;
        if (s->timing) {
            cuda_check(cudaEventRecord(b, s->stream), "event");
            s->pending.emplace_back(a, b);
        }
    });
}

int um_session_set_timing(void* h, int on)
{
    return guarded([&] {
        auto* s = static_cast<SessionBase*>(h);
        s->fold();
        s->timing = on != 0;
    });
}

// Waits for the stream; launches of metropolis_sweeps and their event time
// (timed launches only) since the last reset; throws if a barrier wait ran out.
int um_session_stats(void* h, std::uint64_t* launches, double* ms, int reset)
{
    return guarded([&] {
        auto* s = static_cast<SessionBase*>(h);
        s->fold();
        s->check();
        *launches = s->launches;
        *ms = s->timed_ms;
        if (reset) {
            s->launches = 0;
            s->timed_ms = 0.0;
        }
    });
}

// Total energy (sum of energy_at / 2, FP64) of the current field.
int um_session_energy(void* h, double* e)
{
    return guarded([&] { *e = static_cast<SessionBase*>(h)->energy(); });
}

// Sizes of the Wolff flips since the last call (at most cap; *n = how many
// there were); nothing for Metropolis sessions.
int um_session_take_sizes(void* h, std::uint64_t* out, std::uint64_t cap, std::uint64_t* n)
{
    return guarded([&] {
        const auto s = static_cast<SessionBase*>(h)->take_sizes();
        *n = s.size();
        for (std::size_t k = 0; k < s.size() && k < cap; ++k) out[k] = s[k];
    });
}

int um_session_counters(void* h, std::uint64_t* sweeps, std::uint32_t* grid)
{
    return guarded([&] {
        auto* s = static_cast<SessionBase*>(h);
        *sweeps = s->sweeps();
        *grid = s->grid();
    });
}

}  // extern "C"
