// Device colouring (exact sequential-greedy result, computed in parallel).
#pragma once
#include "world.cuh"

namespace cc {

constexpr uint32_t kMaxColors = 4096;

struct ColorView {
    uint32_t n;
    const uint32_t* lo_off;  // [n+1] lower-index neighbours of the material graph
    const uint32_t* lo;
    ContactsView contacts;
    int grab_active;
    uint32_t grab_v[3];
};

class Coloring {
   public:
    void init(uint32_t n, cudaStream_t s);
    // Recompute the colouring for the current graph, starting from the last one.
    void compute(const ColorView& view, cudaStream_t s);
    uint32_t n_colors() const { return n_colors_; }
    const std::vector<uint32_t>& offsets() const { return offsets_h_; }
    const uint32_t* order() const { return order_.ptr; }
    const uint16_t* colors() const { return cur_; }
    // device word that receives DERR_SORT_WAIT if the colour sort's wait gives up
    void set_error_word(unsigned int* w) { error_word_ = w; }
    size_t last_iterations() const { return last_iterations_; }
    void download(std::vector<uint32_t>& colors);
    uint64_t launches() const { return launches_; }

   private:
    static constexpr int kBatch = 8;
    uint32_t n_ = 0;
    DBuf<uint16_t> a_, b_;
    uint16_t* cur_ = nullptr;
    DBuf<uint32_t> order_, counts_, iota_;
    RadixSorter sorter_;
    unsigned int* error_word_ = nullptr;  // receives DERR_SORT_WAIT (set_error_word)
    DBuf<unsigned int> changed_;
    Pinned<unsigned int> changed_h_;
    Pinned<uint32_t> counts_h_;
    std::vector<uint32_t> offsets_h_;
    uint32_t n_colors_ = 0;
    size_t last_iterations_ = 0;
    uint64_t launches_ = 0;
};

}  // namespace cc
