// simt_host.cpp -- fiber scheduler behind simt_host.hpp (test infrastructure).
#include "simt_host.hpp"

#include <omp.h>

#if !defined(__x86_64__)
#error "simt_host: the fiber switch is written for x86-64 only"
#endif

// Save the callee-saved registers of the running context on its stack, store
// its stack pointer in *save_sp, then resume the context whose stack pointer is
// load_sp.  A fresh fiber stack is laid out so that the final `ret` enters
// fiber_entry with the ABI's call alignment.
asm(R"(
    .text
    .globl simt_switch
    .type simt_switch,@function
simt_switch:
    pushq %rbp
    pushq %rbx
    pushq %r12
    pushq %r13
    pushq %r14
    pushq %r15
    movq %rsp, (%rdi)
    movq %rsi, %rsp
    popq %r15
    popq %r14
    popq %r13
    popq %r12
    popq %rbx
    popq %rbp
    ret
    .size simt_switch, .-simt_switch
)");

namespace simt {

namespace {

constexpr size_t kStackBytes = 128 * 1024;

struct StackPool {
    std::vector<char*> stacks;
    ~StackPool() { for (char* s : stacks) std::free(s); }
    char* get(size_t i) {
        while (stacks.size() <= i) {
            char* s = static_cast<char*>(std::aligned_alloc(64, kStackBytes));
            if (!s) { std::fprintf(stderr, "simt: out of memory for fiber stacks\n"); std::abort(); }
            stacks.push_back(s);
        }
        return stacks[i];
    }
};

StackPool& pool() {
    static thread_local StackPool p;
    return p;
}

[[noreturn]] void fiber_entry() {
    BlockRun* run = current_block();
    (*run->body)();
    run = current_block();
    Fiber& f = run->fibers[run->cur];
    f.state = 2;
    simt_switch(&f.sp, run->sched_sp);
    std::abort();  // a finished fiber is never resumed
}

void* init_stack(char* base) {
    uintptr_t top = reinterpret_cast<uintptr_t>(base + kStackBytes) & ~uintptr_t(15);
    void** sp = reinterpret_cast<void**>(top);
    *--sp = nullptr;                                       // fake return address of fiber_entry
    *--sp = reinterpret_cast<void*>(&fiber_entry);         // `ret` target
    for (int k = 0; k < 6; ++k) *--sp = nullptr;           // rbp rbx r12 r13 r14 r15
    return sp;
}

void run_block(BlockRun& run) {
    const unsigned nthreads = run.bdim.x * run.bdim.y * run.bdim.z;
    run.fibers.resize(nthreads);
    for (unsigned t = 0; t < nthreads; ++t) {
        Fiber& f = run.fibers[t];
        f.state = 0;
        f.tid.x = t % run.bdim.x;
        f.tid.y = (t / run.bdim.x) % run.bdim.y;
        f.tid.z = t / (run.bdim.x * run.bdim.y);
        f.sp = init_stack(pool().get(t));
    }
    current_block() = &run;
    for (;;) {
        bool live = false;
        for (unsigned t = 0; t < nthreads; ++t) {
            Fiber& f = run.fibers[t];
            if (f.state != 0) continue;
            run.cur = static_cast<int>(t);
            simt_switch(&run.sched_sp, f.sp);
        }
        for (unsigned t = 0; t < nthreads; ++t) {
            Fiber& f = run.fibers[t];
            if (f.state == 1) { f.state = 0; live = true; }
        }
        if (!live) break;
    }
    run.cur = -1;
}

}  // namespace

void barrier() {
    BlockRun* run = current_block();
    Fiber& f = run->fibers[run->cur];
    f.state = 1;
    simt_switch(&f.sp, run->sched_sp);
}

void launch(uint3_ grid, uint3_ block, const std::function<void()>& body) {
    const long nblocks = long(grid.x) * grid.y * grid.z;
#pragma omp parallel
    {
        BlockRun run;
        run.body = &body;
        run.bdim = block;
        run.gdim = grid;
#pragma omp for schedule(dynamic, 4)
        for (long b = 0; b < nblocks; ++b) {
            run.bid.x = unsigned(b % grid.x);
            run.bid.y = unsigned((b / grid.x) % grid.y);
            run.bid.z = unsigned(b / (long(grid.x) * grid.y));
            run_block(run);
        }
        current_block() = nullptr;
    }
}

}  // namespace simt
