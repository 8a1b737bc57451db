// Row-shard reducers behind bb_comm: NCCL across processes (one GPU each),
// or an in-process group of shards (several fits' shards on one device,
// driven from one host thread per shard).
#pragma once

#include "grow.cuh"

#include <memory>

struct bb_comm
{
    std::shared_ptr<bb::Reducer> impl;   // shared by a group's members
    std::unique_ptr<bb::Reducer> member; // this participant's view
    bb::Reducer                 *reducer() const
    {
        return member ? member.get() : impl.get();
    }
};
