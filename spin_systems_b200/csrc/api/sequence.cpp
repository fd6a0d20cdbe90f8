// Pulse programs on the device through the C++ core API.
//
// A Sequence's step tree (Evolve / Pulse / Measure / Repeat, the reference's
// include/spinsim/sequence/Sequence.hpp:17-104) is compiled into a flat
// instruction list -- the same linearised form the C ABI's ss_step arrays
// and the batched engine's programs use -- and executed by a program counter
// with an explicit stack of loop frames.  Behaviour follows the reference's
// interpreter (src/sequence/Sequence.cpp:35-106): an Evolve propagates the
// state and then the reference with the same expansion, under its field
// table when it has one; a Pulse rotates both; a Measure records every
// observable's values at the current time.
#include <cstdint>
#include <stdexcept>

#include "spinsim/sequence/Sequence.hpp"

namespace spinsim {
namespace {

// One instruction of a compiled program.
struct Instr {
  enum Kind : std::uint8_t { kEvolve, kPulse, kMeasure, kLoop } kind;
  const Step* step;        // the source step (Evolve or Pulse)
  std::size_t count = 0;   // kLoop: iterations
  std::size_t extent = 0;  // kLoop: instructions in the body that follows
};

void compile(const std::vector<Step>& steps, std::vector<Instr>& program) {
  for (const Step& step : steps) {
    if (std::holds_alternative<Evolve>(step)) {
      program.push_back({Instr::kEvolve, &step});
    } else if (std::holds_alternative<Pulse>(step)) {
      program.push_back({Instr::kPulse, &step});
    } else if (std::holds_alternative<Measure>(step)) {
      program.push_back({Instr::kMeasure, &step});
    } else {
      const Repeat& r = std::get<Repeat>(step);
      const std::size_t at = program.size();
      program.push_back({Instr::kLoop, &step, r.count, 0});
      compile(r.body, program);
      program[at].extent = program.size() - at - 1;
    }
  }
}

std::vector<Instr> compiled(const std::vector<Step>& steps) {
  std::vector<Instr> program;
  compile(steps, program);
  return program;
}

// An Evolve step's field table, installed in the Hamiltonian for the scope's
// lifetime and replaced by the previous fields when it ends (also when the
// propagation throws).  A table wider than the system -- a realisation drawn
// smaller than the configured size -- applies to the system's spins.
class FieldOverride {
 public:
  FieldOverride(Hamiltonian& h, const std::vector<Field>& table) : h_(h) {
    if (table.empty()) return;
    if (table.size() < h.nspins()) {
      throw std::invalid_argument("step field table does not match the number of spins");
    }
    saved_ = h.fields();
    for (SpinIndex s = 0; s < h.nspins(); ++s) h.setField(s, table[s]);
  }
  ~FieldOverride() {
    for (SpinIndex s = 0; s < saved_.size(); ++s) h_.setField(s, saved_[s]);
  }
  FieldOverride(const FieldOverride&) = delete;
  FieldOverride& operator=(const FieldOverride&) = delete;

 private:
  Hamiltonian& h_;
  std::vector<Field> saved_;
};

class Interpreter {
 public:
  explicit Interpreter(RunContext& ctx) : ctx_(ctx) {
    if (ctx.hamiltonian == nullptr || ctx.state == nullptr || ctx.reference == nullptr ||
        ctx.propagator == nullptr) {
      throw std::invalid_argument("run context is missing a required component");
    }
  }

  void execute(const std::vector<Instr>& program) {
    struct Frame {
      std::size_t begin, end, left;  // body [begin, end), iterations still to run
    };
    std::vector<Frame> loops;
    std::size_t pc = 0;
    while (pc < program.size() || !loops.empty()) {
      if (!loops.empty() && pc == loops.back().end) {  // end of a loop body
        if (--loops.back().left > 0) {
          pc = loops.back().begin;
        } else {
          loops.pop_back();
        }
        continue;
      }
      const Instr& in = program[pc++];
      switch (in.kind) {
        case Instr::kEvolve: evolve(std::get<Evolve>(*in.step)); break;
        case Instr::kPulse: pulse(std::get<Pulse>(*in.step)); break;
        case Instr::kMeasure: measure(); break;
        case Instr::kLoop:
          if (in.count == 0 || in.extent == 0) {
            pc += in.extent;  // nothing to repeat
          } else {
            loops.push_back({pc, pc + in.extent, in.count});
          }
          break;
      }
    }
  }

 private:
  void evolve(const Evolve& e) {
    const double tau = e.tauFromDraw ? e.tau * ctx_.tauDraw : e.tau;
    {
      const FieldOverride scope(*ctx_.hamiltonian, e.fields);
      for (StateVector* v : {ctx_.state, ctx_.reference}) {
        ctx_.propagator->evolve(*ctx_.hamiltonian, e.mode, *v, tau, e.nsteps, e.autonormalize);
      }
    }
    ctx_.time += tau * static_cast<double>(e.nsteps);
  }

  void pulse(const Pulse& p) {
    // A rotation of every configured spin rotates every spin of a
    // realisation drawn smaller than the configuration.
    const std::vector<SpinIndex>& t = p.rotation.targets();
    const std::size_t L = ctx_.state->nspins();
    bool every = t.size() > L;
    for (std::size_t i = 0; every && i < t.size(); ++i) every = t[i] == i;
    const SpinRotation narrowed =
        every ? SpinRotation::onAllSpins(p.rotation.axis(), p.rotation.angle(), L) : p.rotation;
    narrowed.apply(*ctx_.state);
    narrowed.apply(*ctx_.reference);
  }

  void measure() {
    if (ctx_.recorder == nullptr) return;
    MeasureContext mc;
    mc.time = ctx_.time;
    mc.state = ctx_.state;
    mc.reference = ctx_.reference;
    mc.hamiltonian = ctx_.hamiltonian;
    mc.subsystemSize = ctx_.subsystemSize;
    std::size_t width = 0;
    for (const auto& o : ctx_.observables) width += o->width();
    row_.assign(width, 0.0);
    std::span<double> rest(row_);
    for (const auto& o : ctx_.observables) {
      o->measure(mc, rest.first(o->width()));
      rest = rest.subspan(o->width());
    }
    ctx_.recorder->record(ctx_.time, row_);
  }

  RunContext& ctx_;
  std::vector<double> row_;
};

}  // namespace

void Sequence::run(RunContext& ctx) const {
  Interpreter(ctx).execute(compiled(steps_));
}

std::size_t Sequence::measurementCount() const {
  // Each Measure counts once per iteration of every loop around it.
  const std::vector<Instr> program = compiled(steps_);
  std::size_t total = 0;
  std::vector<std::pair<std::size_t, std::size_t>> open;  // (end, multiplier)
  std::size_t mult = 1;
  for (std::size_t pc = 0; pc < program.size(); ++pc) {
    while (!open.empty() && pc >= open.back().first) {
      mult = open.back().second;
      open.pop_back();
    }
    if (program[pc].kind == Instr::kMeasure) total += mult;
    if (program[pc].kind == Instr::kLoop) {
      open.emplace_back(pc + 1 + program[pc].extent, mult);
      mult *= program[pc].count;
    }
  }
  return total;
}

std::vector<std::string> resultColumns(std::span<const std::unique_ptr<Observable>> observables) {
  std::vector<std::string> names(1, "time");
  for (const auto& o : observables) {
    std::vector<std::string> own = o->columns();
    names.insert(names.end(), std::make_move_iterator(own.begin()),
                 std::make_move_iterator(own.end()));
  }
  return names;
}

}  // namespace spinsim
