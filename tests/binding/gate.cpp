// The drop-in check: the reference's own Solver (src/field/Solver.cpp), with its CUDA backend replaced by the B200 one
// (online-physics-cuda_b200/binding/B200Solver.cpp, reached through Solver::use_gpu), against the reference's own CPU
// Solver on the same law and state. Built by `make -C oracle binding` against the reference's headers and objects;
// run by tests/test_binding_gpu.py on a machine with a B200.
//
//   b200_gate parity LAW --grid NX NY NZ H --dt DT --steps N --tol T [--init DIR] [--learned]
//       CPU and B200 solvers from the same start (DIR/FIELD.bin, float32 x fastest, else the fields' init values):
//       worst relative difference of every field after N steps within T, the same substeps, violations on both or
//       neither, and two B200 runs equal to the bit.
//   b200_gate world DIR
//       the reference's shipped laws and scene (DIR/world.law, magic.law, fire_test.scene), 12 steps of 0.25 s,
//       within its own gate (1e-4), two B200 runs equal to the bit, the step profiled.
//   b200_gate ops
//       every op alone on a 20 x 14 x 9 lattice, 4 steps, within 2e-5 of the CPU.
//   b200_gate window
//       a window moved three times (only the arriving boxes sent) equals, to the bit, the same window uploaded whole
//       after each move, and stays within 1e-5 of the CPU solver moved the same way.
//   b200_gate lazy
//       lazy readback with an edit between steps gives the bits that fetching every step gives, moving fewer bytes.
//   b200_gate bounds
//       a term that waits for a growing field to pass a threshold starts on the same step on the CPU, eagerly and
//       lazily on the B200 (the idle-term bounds are never short).
//
// One JSON line a check ({"check", "ok", ...}); exit status 0 when every check held.
#include "field/Grid.hpp"
#include "field/Law.hpp"
#include "field/Scene.hpp"
#include "field/Solver.hpp"
#include "field/cuda/CudaSolver.hpp"

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <map>
#include <optional>
#include <sstream>
#include <string>
#include <utility>
#include <vector>

using namespace fieldengine::field;

namespace {

int failures = 0;

void report(const std::string& name, bool ok, const std::string& extra = "")
{
    failures += ok ? 0 : 1;
    std::cout << "{\"check\": \"" << name << "\", \"ok\": " << (ok ? "true" : "false") << (extra.empty() ? "" : ", ") << extra << "}" << std::endl;
}

std::string num(const char* key, double v)
{
    char buf[96];
    std::snprintf(buf, sizeof(buf), "\"%s\": %.9g", key, v);
    return buf;
}

std::optional<Law> compile_text(const std::vector<LawSource>& sources)
{
    CompileResult r = compile_law(sources);
    for (const std::string& e : r.errors) std::cerr << e << "\n";
    return r.law;
}

std::optional<Law> compile_files(const std::vector<std::string>& paths)
{
    std::vector<LawSource> sources;
    for (const std::string& p : paths) {
        std::optional<LawSource> s = read_law_file(p);
        if (!s) {
            std::cerr << "cannot read " << p << "\n";
            return std::nullopt;
        }
        sources.push_back(*s);
    }
    return compile_text(sources);
}

// max |a - b| over a field / max |b| (at least 1e-6), the worst over the fields.
double worst(const FieldSet& got, const FieldSet& want)
{
    double out = 0.0;
    for (std::size_t f = 0; f < want.count(); ++f) {
        const std::vector<float>& a = got.values(static_cast<int>(f));
        const std::vector<float>& b = want.values(static_cast<int>(f));
        double most = 0.0, scale = 1e-6;
        for (std::size_t i = 0; i < b.size(); ++i) {
            most = std::max(most, std::abs(static_cast<double>(a[i]) - static_cast<double>(b[i])));
            scale = std::max(scale, std::abs(static_cast<double>(b[i])));
        }
        out = std::max(out, most / scale);
    }
    return out;
}

bool on_b200(Solver& s)
{
    std::string why;
    if (!s.use_gpu(why)) {
        report("use_gpu", false, "\"why\": \"" + why + "\"");
        return false;
    }
    return true;
}

// ---- parity ------------------------------------------------------------------------------------------------------------

int parity(int argc, char** argv)
{
    if (argc < 3) return 2;
    const std::string path = argv[2];
    GridShape g{8, 8, 8, 1.0};
    double dt = 0.01, tol = 1e-4;
    int steps = 1;
    bool learned = false;
    std::string init;
    for (int i = 3; i < argc; ++i) {
        const std::string a = argv[i];
        if (a == "--grid" && i + 4 < argc) {
            g = GridShape{std::atoi(argv[i + 1]), std::atoi(argv[i + 2]), std::atoi(argv[i + 3]), std::atof(argv[i + 4])};
            i += 4;
        } else if (a == "--dt" && i + 1 < argc) dt = std::atof(argv[++i]);
        else if (a == "--steps" && i + 1 < argc) steps = std::atoi(argv[++i]);
        else if (a == "--tol" && i + 1 < argc) tol = std::atof(argv[++i]);
        else if (a == "--init" && i + 1 < argc) init = argv[++i];
        else if (a == "--learned") learned = true;
    }
    const std::optional<Law> law = compile_files({path});
    if (!law) {
        report("compiles", false);
        return 1;
    }
    Solver cpu(*law, g), b200(*law, g), again(*law, g);
    for (Solver* s : {&cpu, &b200, &again}) {
        FieldSet& f = s->fields();
        for (std::size_t id = 0; id < f.count() && !init.empty(); ++id) {
            std::ifstream in(init + "/" + f.at(static_cast<int>(id)).name + ".bin", std::ios::binary);
            if (!in) continue;
            std::vector<float>& v = f.values(static_cast<int>(id));
            in.read(reinterpret_cast<char*>(v.data()), static_cast<std::streamsize>(v.size() * sizeof(float)));
        }
        s->set_learned(learned);
        s->refresh_derived();
    }
    if (!on_b200(b200) || !on_b200(again)) return 1;
    bool same_substeps = true, same_violations = true;
    for (int k = 0; k < steps; ++k) {
        cpu.step(dt);
        b200.step(dt);
        again.step(dt);
        same_substeps = same_substeps && cpu.last_substeps() == b200.last_substeps();
        same_violations = same_violations && cpu.violations().empty() == b200.violations().empty();
    }
    const double w = worst(std::as_const(b200).fields(), std::as_const(cpu).fields());
    report("parity", w <= tol && same_substeps && same_violations,
        num("worst", w) + ", " + num("tol", tol) + ", \"same_substeps\": " + (same_substeps ? "true" : "false") +
            ", \"same_violations\": " + (same_violations ? "true" : "false") + ", \"backend\": \"" + b200.backend_api() + "\"");
    report("deterministic", std::as_const(b200).fields().digest() == std::as_const(again).fields().digest());
    return 0;
}

// ---- the reference's shipped laws ---------------------------------------------------------------------------------------

int world(const std::string& dir)
{
    Scene scene;
    std::string error;
    // The scene names its laws by repository path (assets/law/...): read them from `dir` instead.
    if (!load_scene(dir + "/fire_test.scene", scene, error)) {
        report("world scene", false, "\"why\": \"" + error + "\"");
        return 1;
    }
    const std::optional<Law> law = compile_files({dir + "/world.law", dir + "/magic.law"});
    if (!law) {
        report("world compiles", false);
        return 1;
    }
    Solver cpu(*law, scene.grid), b200(*law, scene.grid), again(*law, scene.grid);
    for (Solver* s : {&cpu, &b200, &again}) {
        if (!apply_scene(scene, *s, error)) {
            report("world scene applies", false, "\"why\": \"" + error + "\"");
            return 1;
        }
    }
    if (!on_b200(b200) || !on_b200(again)) return 1;
    for (int k = 0; k < 12; ++k) {
        cpu.step(0.25);
        b200.step(0.25);
        again.step(0.25);
    }
    const double w = worst(std::as_const(b200).fields(), std::as_const(cpu).fields());
    report("world law within the reference's gate", w < 1e-4, num("worst", w) + ", \"cells\": " + std::to_string(scene.grid.cells()));
    report("world law: two B200 runs equal to the bit", std::as_const(b200).fields().digest() == std::as_const(again).fields().digest());
    report("world law: the same contracts break or hold", b200.violations().empty() == cpu.violations().empty());
    const StepProfile& p = b200.profile();
    report("world law: the step is profiled", p.launches > 0, num("gpu_ms", p.gpu_ms) + ", \"launches\": " + std::to_string(p.launches));
    return 0;
}

// ---- every op alone ---------------------------------------------------------------------------------------------------------

void paint(FieldSet& f, const GridShape& g)
{
    for (int z = 0; z < g.nz; ++z) {
        for (int y = 0; y < g.ny; ++y) {
            for (int x = 0; x < g.nx; ++x) {
                const std::size_t i = g.index(x, y, z);
                f.values(0)[i] = static_cast<float>(0.5 + 0.45 * std::cos(0.9 * x - 0.4 * y + 0.2 * z));
                if (f.count() > 1) f.values(1)[i] = ((3 * x + y + 5 * z) % 5) < 2 ? 1.0f : 0.0f;
            }
        }
    }
}

int ops()
{
    const char* rates[] = {
        "lap(A)", "gx(A) - gy(A) + gz(A)", "diffuse(0.25 + B, A)", "adv(A, B - 0.4, -0.2, 0.3)", "fall(A, B, 1.5)",
        "spread(A, B, 0.4)", "topple(A, B, 0.8)", "shift(A, -1, 2, 0) - A", "shift_t(A, 1, 0, -1) - A",
        "pos(A - 0.4) * sqrt(abs(B - A)) - clamp(A, 0.3, 0.6) + min(A, B) * max(A, 0.2)", "abs(B - 0.3) ^ 1.5 - exp(-A) + log(2 + B)",
        "0.02 * (maxof(A) - minof(B)) + 0.0002 * sumof(A)", "0.05 * distance(B)", "0.05 * poisson(B - 0.4, 12)",
        "tridiag_x(-0.2 * (1 + B), 1.5 + A, -0.2, A) - A",
    };
    const GridShape g{20, 14, 9, 0.5};
    for (const char* rate : rates) {
        const std::string text = std::string("field A init 0 range -1e9 1e9\nfield B init 0 range -1e9 1e9\nterm t\n  d A = ") + rate + "\n";
        const std::optional<Law> law = compile_text({LawSource{"op", text}});
        if (!law) {
            report(std::string("op compiles: ") + rate, false);
            continue;
        }
        Solver cpu(*law, g), b200(*law, g);
        paint(cpu.fields(), g);
        paint(b200.fields(), g);
        if (!on_b200(b200)) return 1;
        for (int k = 0; k < 4; ++k) {
            cpu.step(0.02);
            b200.step(0.02);
        }
        const double w = worst(std::as_const(b200).fields(), std::as_const(cpu).fields());
        report(std::string("op: ") + rate, w < 2e-5, num("worst", w));
    }
    return 0;
}

// ---- a moved window -----------------------------------------------------------------------------------------------------------

int window()
{
    const std::string text = "field A init 0 range -1e9 1e9\nfield B init 0 range -1e9 1e9\nterm t\n  d A = diffuse(0.3, A) - 0.1 * gx(B)\n"
                             "  conserves A\nterm u\n  d B = 0.2 * lap(B) + 0.05 * A\nderive D = distance(B)\n";
    const std::optional<Law> law = compile_text({LawSource{"window", text}});
    if (!law) {
        report("window law compiles", false);
        return 1;
    }
    const GridShape g{40, 24, 12, 1.0};
    Solver ring(*law, g), whole(*law, g), cpu(*law, g);
    // What the world holds at lattice cell (x, y, z) when the window starts at (ox, oy, oz).
    auto world_value = [](int field, int x, int y, int z) {
        const std::uint32_t h = (static_cast<std::uint32_t>(x) * 73856093u) ^ (static_cast<std::uint32_t>(y) * 19349663u) ^
            (static_cast<std::uint32_t>(z) * 83492791u) ^ (static_cast<std::uint32_t>(field) * 2654435761u);
        return field == 0 ? static_cast<float>((h & 1023u) / 1023.0) : ((h >> 10) & 7u) < 3u ? 1.0f : 0.0f;
    };
    auto fill = [&](FieldSet& f, int ox, int oy, int oz, const CellBox& b) {
        for (int field = 0; field < 2; ++field) {
            for (int z = b.z0; z < b.z1; ++z) {
                for (int y = b.y0; y < b.y1; ++y) {
                    for (int x = b.x0; x < b.x1; ++x) f.values(field)[g.index(x, y, z)] = world_value(field, x + ox, y + oy, z + oz);
                }
            }
        }
    };
    for (Solver* s : {&ring, &whole, &cpu}) {
        fill(s->fields(), 0, 0, 0, CellBox{0, 0, 0, g.nx, g.ny, g.nz});
        s->refresh_derived();
    }
    if (!on_b200(ring) || !on_b200(whole)) return 1;
    for (Solver* s : {&ring, &whole, &cpu}) s->step(0.05);
    int ox = 0, oy = 0, oz = 0;
    const int moves[3][3] = {{6, 0, 0}, {0, -5, 0}, {-3, 4, 2}};
    for (const auto& m : moves) {
        const int dx = m[0], dy = m[1], dz = m[2];
        ox += dx;
        oy += dy;
        oz += dz;
        // The cells that arrive: the slabs of the new window not inside the old one.
        std::vector<CellBox> arriving;
        if (dx > 0) arriving.push_back(CellBox{g.nx - dx, 0, 0, g.nx, g.ny, g.nz});
        if (dx < 0) arriving.push_back(CellBox{0, 0, 0, -dx, g.ny, g.nz});
        if (dy > 0) arriving.push_back(CellBox{0, g.ny - dy, 0, g.nx, g.ny, g.nz});
        if (dy < 0) arriving.push_back(CellBox{0, 0, 0, g.nx, -dy, g.nz});
        if (dz > 0) arriving.push_back(CellBox{0, 0, g.nz - dz, g.nx, g.ny, g.nz});
        if (dz < 0) arriving.push_back(CellBox{0, 0, 0, g.nx, g.ny, -dz});
        for (Solver* s : {&ring, &whole, &cpu}) {
            FieldSet& f = s == &ring ? s->shift_window(dx, dy, dz, arriving) : s->fields();
            // Slide what stays (the cell now at c was at c + d), then paint what arrived.
            for (int field = 0; field < 2; ++field) {
                const std::vector<float> old = f.values(field);
                for (int z = 0; z < g.nz; ++z) {
                    for (int y = 0; y < g.ny; ++y) {
                        for (int x = 0; x < g.nx; ++x) {
                            if (g.inside(x + dx, y + dy, z + dz)) f.values(field)[g.index(x, y, z)] = old[g.index(x + dx, y + dy, z + dz)];
                        }
                    }
                }
            }
            for (const CellBox& b : arriving) fill(f, ox, oy, oz, b);
            s->refresh_derived();
            s->step(0.05);
        }
    }
    const std::uint64_t a = std::as_const(ring).fields().digest(), b = std::as_const(whole).fields().digest();
    report("a window moved on the card (only the arriving boxes sent) is to the bit the window sent whole", a == b,
        "\"upload_bytes_last\": " + std::to_string(ring.profile().upload_bytes));
    const double w = worst(std::as_const(ring).fields(), std::as_const(cpu).fields());
    report("the moved window holds to the CPU solver moved the same way", w < 1e-5, num("worst", w));
    return 0;
}

// ---- lazy readback --------------------------------------------------------------------------------------------------------------

int lazy()
{
    const std::string text = "field T init 300 range 0 1e6\nfield F init 0 range 0 1\nparam k = 0.8\nterm heat\n  d T = diffuse(k, T) + 40 * F\n"
                             "  conserves T\nterm burn\n  d F = -0.3 * F * step(T - 310)\nderive G = gx(T) * gx(T) + gy(T) * gy(T)\n";
    const std::optional<Law> law = compile_text({LawSource{"lazy", text}});
    if (!law) {
        report("lazy law compiles", false);
        return 1;
    }
    const GridShape g{48, 32, 16, 0.5};
    Solver eager(*law, g), lazy_s(*law, g);
    for (Solver* s : {&eager, &lazy_s}) {
        FieldSet& f = s->fields();
        for (std::size_t i = 0; i < g.cells(); ++i) f.values(1)[i] = ((i * 2654435761u) >> 7) % 9 == 0 ? 1.0f : 0.0f;
        if (!on_b200(*s)) return 1;
    }
    lazy_s.set_lazy_readback(true);
    const int T = lazy_s.field("T");
    const std::size_t cell = g.index(g.nx / 2, g.ny / 3, g.nz / 2);
    std::size_t eager_bytes = 0, lazy_bytes = 0;
    for (int k = 0; k < 20; ++k) {
        if (k == 11) {
            eager.edit_cell(T, cell) += 250.0f;
            lazy_s.edit_cell(T, cell) += 250.0f;
        }
        eager.step(0.02);
        lazy_s.step(0.02);
        eager_bytes += eager.profile().download_bytes;
        lazy_bytes += lazy_s.profile().download_bytes;
    }
    report("lazy readback moves less than fetching every step", lazy_bytes < eager_bytes,
        "\"lazy_bytes\": " + std::to_string(lazy_bytes) + ", \"eager_bytes\": " + std::to_string(eager_bytes));
    report("lazy readback with an edit between steps gives the bits of fetching every step",
        std::as_const(lazy_s).fields().digest() == std::as_const(eager).fields().digest());
    return 0;
}

// ---- carried bounds ---------------------------------------------------------------------------------------------------------------

int bounds()
{
    // Y counts the steps X is past thr; its term is idle while X's bounds say X is below.
    const std::pair<const char*, std::string> cases[] = {
        {"a field grown in substeps", "field X init 1 range 0 1e30\nfield Y init 0 range 0 1e9\nparam a = 3\nparam thr = 20000\n"
                                      "term grow\n  d X = a * X\n  max_dt = 0.08 / a\nterm over\n  d Y = step(X - thr)\n"},
        {"a field past its unclamped range", "field X init 1 range 0 50\nfield Y init 0 range 0 1e9\nparam thr = 400\n"
                                             "term grow\n  d X = 0.6 * X\nterm over\n  d Y = step(X - thr)\n"},
    };
    for (const auto& [what, text] : cases) {
        std::vector<float> y[3];
        for (int mode = 0; mode < 3; ++mode) {
            const std::optional<Law> law = compile_text({LawSource{"bounds", text}});
            if (!law) return 1;
            Solver s(*law, GridShape{8, 8, 2, 1.0});
            if (mode > 0 && !on_b200(s)) return 1;
            s.set_lazy_readback(mode == 2);
            for (int k = 0; k < 14; ++k) s.step(1.0);
            y[mode] = std::as_const(s).values(s.field("Y"));
        }
        report(std::string("bounds, ") + what + ": the waiting term starts when the CPU's does, eagerly and lazily",
            !y[0].empty() && y[0][0] > 0.f && y[1] == y[0] && y[2] == y[0], num("Y_cpu", y[0].empty() ? -1 : y[0][0]) + ", " +
                num("Y_eager", y[1].empty() ? -1 : y[1][0]) + ", " + num("Y_lazy", y[2].empty() ? -1 : y[2][0]));
    }
    return 0;
}

} // namespace

int main(int argc, char** argv)
{
    setenv("FIELD_BACKEND", "cuda", 1); // Solver::use_gpu: the CUDA backend (this one) or nothing
    if (argc < 2) {
        std::cerr << "usage: b200_gate parity|world|ops|window|lazy|bounds ...\n";
        return 2;
    }
    const std::string mode = argv[1];
    if (const std::string why = CudaSolver::unavailable(); !why.empty()) {
        report("device", false, "\"why\": \"" + why + "\"");
        return 1;
    }
    int rc = 2;
    if (mode == "parity") rc = parity(argc, argv);
    else if (mode == "world" && argc > 2) rc = world(argv[2]);
    else if (mode == "ops") rc = ops();
    else if (mode == "window") rc = window();
    else if (mode == "lazy") rc = lazy();
    else if (mode == "bounds") rc = bounds();
    if (rc == 2) std::cerr << "unknown mode or missing arguments\n";
    return rc != 0 ? rc : (failures == 0 ? 0 : 1);
}
