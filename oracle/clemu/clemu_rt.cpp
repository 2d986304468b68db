// clemu_rt.cpp -- fiber scheduler of the CPU work-group emulator (x86-64 SysV).
// TEST INFRASTRUCTURE ONLY.  A fiber switch saves the callee-saved registers,
// MXCSR and the x87 control word, then swaps stack pointers.
#include "clemu_rt.hpp"

#include <cstdio>
#include <cstdlib>
#include <vector>

extern "C" void clemu_swap(void** save_sp, void* load_sp);
asm(R"(
.text
.globl clemu_swap
.hidden clemu_swap
.type clemu_swap,@function
clemu_swap:
    pushq %rbp
    pushq %rbx
    pushq %r12
    pushq %r13
    pushq %r14
    pushq %r15
    subq $8, %rsp
    stmxcsr (%rsp)
    fnstcw 4(%rsp)
    movq %rsp, (%rdi)
    movq %rsi, %rsp
    ldmxcsr (%rsp)
    fldcw 4(%rsp)
    addq $8, %rsp
    popq %r15
    popq %r14
    popq %r13
    popq %r12
    popq %rbx
    popq %rbp
    ret
.size clemu_swap,.-clemu_swap
)");

namespace clemu {
namespace {

const size_t kStack = 256 * 1024;

struct Fiber {
    void* sp = nullptr;
    char* stack = nullptr;
    int done = 0;
};

struct Group {
    std::vector<Fiber> f;
    void* sched_sp = nullptr;
    int cur = 0;
    int n = 0;
    size_t gid = 0;
    const std::function<void()>* body = nullptr;
};

thread_local Group* tl_group = nullptr;

void fiber_entry()
{
    Group* g = tl_group;
    (*g->body)();
    g->f[g->cur].done = 1;
    clemu_swap(&g->f[g->cur].sp, g->sched_sp);
    std::abort();  // a finished fiber is never resumed
}

void init_fiber(Fiber& fb)
{
    if (!fb.stack) fb.stack = (char*)std::aligned_alloc(64, kStack);
    uintptr_t top = ((uintptr_t)fb.stack + kStack) & ~(uintptr_t)15;
    uint64_t* sp = (uint64_t*)top;
    *--sp = 0;                               // pad: rsp after the entry `ret` is 8 mod 16
    *--sp = (uint64_t)(uintptr_t)&fiber_entry;  // return address
    for (int i = 0; i < 6; ++i) *--sp = 0;   // rbp rbx r12 r13 r14 r15
    uint32_t mx = 0;
    uint16_t cw = 0;
    asm volatile("stmxcsr %0" : "=m"(mx));
    asm volatile("fnstcw %0" : "=m"(cw));
    uint64_t ctl = (uint64_t)mx | ((uint64_t)cw << 32);
    *--sp = ctl;
    fb.sp = sp;
    fb.done = 0;
}

}  // namespace

size_t local_id() { return (size_t)tl_group->cur; }
size_t group_id() { return tl_group->gid; }
int local_size() { return tl_group->n; }

void barrier()
{
    Group* g = tl_group;
    clemu_swap(&g->f[g->cur].sp, g->sched_sp);
}

int launch(size_t groups, int local_size, const std::function<void()>& body)
{
    thread_local Group grp;
    Group* g = &grp;
    if ((int)g->f.size() < local_size) g->f.resize(local_size);
    g->n = local_size;
    g->body = &body;
    Group* prev = tl_group;
    tl_group = g;
    int status = 0;
    for (size_t gid = 0; gid < groups; ++gid) {
        g->gid = gid;
        for (int i = 0; i < local_size; ++i) init_fiber(g->f[i]);
        int remaining = local_size;
        while (remaining > 0) {
            int finished = 0, waiting = 0;
            for (int i = 0; i < local_size; ++i) {
                if (g->f[i].done) continue;
                g->cur = i;
                clemu_swap(&g->sched_sp, g->f[i].sp);
                if (g->f[i].done) { ++finished; --remaining; }
                else ++waiting;
            }
            if (finished && waiting) {  // some work-items left while others wait at a barrier
                status = 1;
                std::fprintf(stderr, "clemu: divergent barrier in group %zu\n", gid);
                break;
            }
        }
        if (status) break;
    }
    tl_group = prev;
    return status;
}

}  // namespace clemu
