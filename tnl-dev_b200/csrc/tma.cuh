// Inline-PTX helpers for Hopper/Blackwell bulk asynchronous copies (TMA
// engine, `cp.async.bulk`) completing on shared-memory mbarriers.
//
// Only the non-tensor, non-multicast form is used: global -> this CTA's own
// shared memory. Every wait is bounded; callers turn a timeout into an error
// flag and a clean exit instead of a hang.
#pragma once

#include <cstdint>

namespace b2s {

__device__ __forceinline__ uint32_t
smem_u32( const void* p )
{
   return static_cast< uint32_t >( __cvta_generic_to_shared( p ) );
}

__device__ __forceinline__ void
mbar_init( uint64_t* bar, uint32_t count )
{
   asm volatile( "mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"( smem_u32( bar ) ), "r"( count ) : "memory" );
}

// make barrier initialisation visible to the async proxy
__device__ __forceinline__ void
fence_mbar_init()
{
   asm volatile( "fence.mbarrier_init.release.cluster;" ::: "memory" );
}

// order earlier generic-proxy accesses of shared memory before later
// async-proxy (bulk copy) writes to the same memory
__device__ __forceinline__ void
fence_proxy_async_smem()
{
   asm volatile( "fence.proxy.async.shared::cta;" ::: "memory" );
}

__device__ __forceinline__ void
mbar_arrive_expect_tx( uint64_t* bar, uint32_t bytes )
{
   asm volatile( "mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"( smem_u32( bar ) ), "r"( bytes )
                 : "memory" );
}

__device__ __forceinline__ void
mbar_arrive( uint64_t* bar )
{
   asm volatile( "mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"( smem_u32( bar ) ) : "memory" );
}

// bulk copy global -> shared; src and dst 16-byte aligned, bytes a multiple of 16
__device__ __forceinline__ void
bulk_g2s( void* dst, const void* src, uint32_t bytes, uint64_t* bar )
{
   asm volatile( "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                    smem_u32( dst ) ),
                 "l"( src ), "r"( bytes ), "r"( smem_u32( bar ) )
                 : "memory" );
}

__device__ __forceinline__ bool
mbar_try_wait( uint64_t* bar, uint32_t parity )
{
   uint32_t ok;
   asm volatile(
      "{\n\t.reg .pred P;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 P, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, P;\n\t}"
      : "=r"( ok )
      : "r"( smem_u32( bar ) ), "r"( parity )
      : "memory" );
   return ok != 0;
}

// Bounded wait on one phase of an mbarrier: false after `limit` failed tries
// (each try may suspend the thread for a short, hardware-chosen time).
constexpr uint32_t kWaitLimit = 1u << 22;

__device__ __forceinline__ bool
mbar_wait_bounded( uint64_t* bar, uint32_t parity, uint32_t limit = kWaitLimit )
{
   for( uint32_t i = 0; i < limit; i++ )
      if( mbar_try_wait( bar, parity ) )
         return true;
   return false;
}

}  // namespace b2s
