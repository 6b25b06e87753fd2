"""Checkers for the rasterizer (test infrastructure, never imported by the product).

reference.py  ctypes access to the reference rasterizer compiled from its own sources
splat_oracle  CPU restatement of the reference algorithm (C, built by the Makefile)
"""
