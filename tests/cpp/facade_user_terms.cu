// A reference-style program whose models use terms written by the user,
// built with nvcc so that the facade's drivers run those terms on the device
// (umc/device_facade.cuh).  Apart from the __host__ __device__ markers on the
// terms, it is what a user of the reference writes: PairModel / CellModel
// over square_lattice / hypercubic_plaquettes, Metropolis and Wolff with the
// reference's proposals and axes, Pcg32 for the keys, data() to read back.
//
// Writes to argv[1], in order: the XY start and end angles; the Ising start
// spins, the spins after 12 flips, their cluster sizes, the spins after one
// more Wolff sweep and the mean cluster size; the U(1) start and end angles;
// the O(3) start and end spins; the SU(3) start and end links (18 doubles
// each, the reference's data() layout).
#include <umc/umc.hpp>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <numbers>
#include <vector>

// E = -J cos(t_i - t_j) on U1Link angles: the XY model as a user pair term.
struct XYAngleTerm
{
    using dtype = U1Link;
    using energy_type = double;
    static constexpr std::size_t arity = 2;
    double J = 1.0;

    __host__ __device__ energy_type energy(const dtype* const* l) const { return -J * cos(l[0]->theta - l[1]->theta); }
    __host__ __device__ energy_type delta(std::size_t which, const dtype* old, const dtype* nw,
                                          const dtype* const* l) const
    {
        const dtype* fixed = l[which == 0 ? 1 : 0];
        return -J * (cos(nw->theta - fixed->theta) - cos(old->theta - fixed->theta));
    }
};

// E = -J s_i s_j on int8 spins, in int32 (IsingTerm's arithmetic, rewritten by the user).
struct MyIsingTerm
{
    using dtype = IsingSpin;
    using energy_type = std::int32_t;
    static constexpr std::size_t arity = 2;
    std::int32_t J = 1;

    __host__ __device__ energy_type energy(const dtype* const* l) const { return -J * (std::int32_t(*l[0]) * *l[1]); }
    __host__ __device__ energy_type delta(std::size_t which, const dtype* old, const dtype* nw,
                                          const dtype* const* l) const
    {
        const dtype* fixed = l[which == 0 ? 1 : 0];
        return -J * (std::int32_t(*nw) * *fixed - std::int32_t(*old) * *fixed);
    }
};

// S_p = beta (1 - cos(t0 + t1 - t2 - t3)) as a user cell term of arity 4.
struct MyPlaquetteTerm
{
    using dtype = U1Link;
    using energy_type = double;
    static constexpr std::size_t arity = 4;
    double beta = 1.0;

    __host__ __device__ static double angle_cos(const double* t) { return cos(t[0] + t[1] - t[2] - t[3]); }
    __host__ __device__ energy_type energy(const dtype* const* l) const
    {
        const double t[4] = {l[0]->theta, l[1]->theta, l[2]->theta, l[3]->theta};
        return beta * (1.0 - angle_cos(t));
    }
    __host__ __device__ energy_type delta(std::size_t which, const dtype*, const dtype* nw,
                                          const dtype* const* l) const
    {
        double t[4] = {l[0]->theta, l[1]->theta, l[2]->theta, l[3]->theta};
        const double before = angle_cos(t);
        t[which] = nw->theta;
        return beta * (before - angle_cos(t));
    }
};

// E = -J s_i . s_j on VectorDof<3>, as a user would write HeisenbergTerm.
struct MyHeisenbergTerm
{
    using dtype = double;
    using energy_type = double;
    static constexpr std::size_t arity = 2;
    double J = 1.0;

    __host__ __device__ static double dot3(const double* a, const double* b)
    {
        return a[0] * b[0] + a[1] * b[1] + a[2] * b[2];
    }
    __host__ __device__ energy_type energy(const dtype* const* l) const { return -J * dot3(l[0], l[1]); }
    __host__ __device__ energy_type delta(std::size_t which, const dtype* old, const dtype* nw,
                                          const dtype* const* l) const
    {
        const dtype* fixed = l[which == 0 ? 1 : 0];
        return -J * (dot3(nw, fixed) - dot3(old, fixed));
    }
};

// S_p = beta (1 - Re Tr(U0 U1 U2^dag U3^dag) / 3) on SULink<3>, written
// against the reference's SULink interface (plaquette, operator*, dagger).
struct MySU3PlaquetteTerm
{
    using dtype = SULink<3>;
    using energy_type = double;
    static constexpr std::size_t arity = 4;
    double beta = 1.0;

    __host__ __device__ energy_type energy(const dtype* const* l) const
    {
        return beta * (1.0 - plaquette(*l[0], *l[1], *l[2], *l[3]));
    }
    __host__ __device__ energy_type delta(std::size_t which, const dtype*, const dtype* nw,
                                          const dtype* const* l) const
    {
        const dtype* p[4] = {l[0], l[1], l[2], l[3]};
        p[which] = nw;
        return beta * (plaquette(*l[0], *l[1], *l[2], *l[3]) - plaquette(*p[0], *p[1], *p[2], *p[3]));
    }
};

static_assert(CellTerm<XYAngleTerm, U1Dof> && CellTerm<MyIsingTerm, IsingDof> && CellTerm<MyPlaquetteTerm, U1Dof> &&
              CellTerm<MyHeisenbergTerm, VectorDof<3>> && CellTerm<MySU3PlaquetteTerm, SUDof<3>>);

template <class T>
static void put(std::FILE* f, const T* p, std::size_t n)
{
    if (std::fwrite(p, sizeof(T), n, f) != n) throw std::runtime_error("write failed");
}

template <class M>
static std::vector<double> angles(const M& m)
{
    std::vector<double> t(m.sites());
    for (std::size_t i = 0; i < m.sites(); ++i) t[i] = m.data()[i].theta;
    return t;
}

int main(int argc, char** argv)
{
    if (argc < 2) return 2;
    std::FILE* out = std::fopen(argv[1], "wb");
    if (!out) return 2;
    try {
        // XY: PairModel<U1Dof, user term, PairGraph<>> with U1Shift, 3 sweeps then 2 observed sweeps
        PairModel<U1Dof, XYAngleTerm, PairGraph<>> xy(square_lattice(32, 32), XYAngleTerm{1.0});
        Pcg32 init(5, 3);
        for (std::size_t i = 0; i < xy.sites(); ++i) {
            const U1Link l{2.0 * std::numbers::pi * init.uni() - std::numbers::pi};
            xy.update(i, &l);
        }
        const auto xy0 = angles(xy);
        {
            Metropolis metro(xy, U1Shift{1.0}, Pcg32(4, 0), 1.1);
            metro.run(3);
            double e = 0.0;
            metro.sample(2, [&](const auto& m) {
                double ek = 0.0;
                for (std::size_t i = 0; i < m.sites(); ++i) ek += 0.5 * m.energy_at(i);
                // the device-recorded energy of this sweep equals the host sum
                const double rec = metro.records()[0];
                if (std::fabs(rec - ek) > 1e-9 * double(m.sites())) throw std::runtime_error("record differs");
                e += ek;
            });
            std::printf("XY user term: E per site after 5 sweeps %.6f\n", e / 2.0 / double(xy.sites()));
        }
        const auto xy1 = angles(xy);
        put(out, xy0.data(), xy0.size());
        put(out, xy1.data(), xy1.size());

        // Ising: PairModel<IsingDof, user term, PairGraph<>>, Wolff with FixedAxis, 12 flips
        PairModel<IsingDof, MyIsingTerm, PairGraph<>> ising(square_lattice(24, 24), MyIsingTerm{1});
        for (std::size_t i = 0; i < ising.sites(); ++i) {
            const IsingSpin s = init.uni() < 0.5 ? IsingSpin(1) : IsingSpin(-1);
            ising.update(i, &s);
        }
        std::vector<IsingSpin> s0(ising.data(), ising.data() + ising.sites());
        std::vector<std::uint64_t> sizes(12);
        std::vector<IsingSpin> s1;
        double mean_after_sweep = 0.0;
        {
            Wolff wolf(ising, FixedAxis{}, Pcg32(13, 0), 0.44);
            wolf.flips(12, sizes.data());
            std::printf("Ising user term: mean cluster %.2f\n", wolf.mean_cluster_size());
            s1.assign(ising.data(), ising.data() + ising.sites());
            wolf.sweep();  // flips 12, 13, ... until the flipped sites cover the lattice
            mean_after_sweep = wolf.mean_cluster_size();
        }
        std::vector<IsingSpin> s2(ising.data(), ising.data() + ising.sites());
        put(out, s0.data(), s0.size());
        put(out, s1.data(), s1.size());
        put(out, sizes.data(), sizes.size());
        put(out, s2.data(), s2.size());
        put(out, &mean_after_sweep, 1);

        // U(1): CellModel<U1Dof, user cell term, CellComplex<4>> on the 4^4 plaquettes, 2 sweeps
        CellModel<U1Dof, MyPlaquetteTerm, CellComplex<4>> u1(hypercubic_plaquettes(4), MyPlaquetteTerm{1.3});
        for (std::size_t i = 0; i < u1.sites(); ++i) {
            const U1Link l{2.0 * std::numbers::pi * init.uni() - std::numbers::pi};
            u1.update(i, &l);
        }
        const auto u0 = angles(u1);
        {
            Metropolis metro(u1, U1Shift{0.7}, Pcg32(9, 0), 1.0);
            metro.run(2);
        }
        const auto u1a = angles(u1);
        std::printf("U(1) user cell term: S = %.6f\n", u1.total_energy());
        put(out, u0.data(), u0.size());
        put(out, u1a.data(), u1a.size());

        // O(3): PairModel<VectorDof<3>, user term, PairGraph<>> on 8^3 with LocalRotation, 2 sweeps
        PairModel<VectorDof<3>, MyHeisenbergTerm, PairGraph<>> o3(cubic_lattice(8, 8, 8), MyHeisenbergTerm{1.0});
        for (std::size_t i = 0; i < o3.sites(); ++i) {
            double v[3];
            UniformSphereN<3>{}.sample(nullptr, init, v);
            o3.update(i, v);
        }
        const std::vector<double> v0(o3.data(), o3.data() + 3 * o3.sites());
        {
            Metropolis metro(o3, LocalRotation<3>{0.6}, Pcg32(21, 0), 0.693);
            metro.run(2);
        }
        const std::vector<double> v1(o3.data(), o3.data() + 3 * o3.sites());
        put(out, v0.data(), v0.size());
        put(out, v1.data(), v1.size());

        // SU(3): CellModel<SUDof<3>, user cell term, CellComplex<4>> on the 4^4
        // plaquettes, the reference's SUShift<3>, 2 sweeps.  Start: each link
        // the identity moved by four wide SUShift steps drawn on the host.
        CellModel<SUDof<3>, MySU3PlaquetteTerm, CellComplex<4>> su(hypercubic_plaquettes(4), MySU3PlaquetteTerm{5.7});
        for (std::size_t i = 0; i < su.sites(); ++i) {
            SULink<3> u = SULink<3>::identity(), w;
            for (int k = 0; k < 4; ++k) {
                SUShift<3>{1.0}.sample(&u, init, &w);
                u = w;
            }
            su.update(i, &u);
        }
        const auto* s0p = reinterpret_cast<const double*>(su.data());
        const std::vector<double> su0(s0p, s0p + 18 * su.sites());
        {
            Metropolis metro(su, SUShift<3>{0.3}, Pcg32(33, 0), 1.0);
            metro.run(2);
        }
        const auto* s1p = reinterpret_cast<const double*>(su.data());
        const std::vector<double> su1(s1p, s1p + 18 * su.sites());
        double worst = 0.0;
        for (std::size_t i = 0; i < su.sites(); ++i) {
            const double e = su.data()[i].unitarity_error();
            worst = e > worst ? e : worst;
        }
        std::printf("SU(3) user cell term: S = %.6f, unitarity error %.2e\n", su.total_energy(), worst);
        put(out, su0.data(), su0.size());
        put(out, su1.data(), su1.size());
    } catch (const std::exception& e) {
        std::fprintf(stderr, "error: %s\n", e.what());
        std::fclose(out);
        return 1;
    }
    std::fclose(out);
    std::printf("ok\n");
    return 0;
}
