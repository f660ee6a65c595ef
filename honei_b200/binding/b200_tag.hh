/*
 * The B200 tag of a HONEI tree: tag-dispatched operators (Product<tags::B200>,
 * Defect<tags::B200>, ...) run on the sm_100a kernels of libhonei_b200 through its
 * C ABI, and containers locked with tags::B200::memory_value live in that GPU's
 * memory.  The tree's honei/util/tags.hh must carry the tag value tv_b200 in its
 * TagValue enum (one line before tv_none; binding.mk builds such a copy of the
 * header for a tree that does not have it yet).
 */
#pragma once
#ifndef HONEI_B200_BINDING_TAG_HH
#define HONEI_B200_BINDING_TAG_HH 1

#include <honei/util/tags.hh>

#include <string>

namespace honei
{
    namespace tags
    {
        /* the same shape as the tree's GPU::CUDA tag (util/tags.hh:183-188) */
        struct B200 :
            public InstantiationPolicy<B200, NonCopyable>
        {
            const static TagValue tag_value = tv_b200;
            const static TagValue memory_value = tv_b200;
            const static std::string name;
        };
    }
}

#endif
