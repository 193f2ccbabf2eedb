"""Argument types of the fault / driver entry points (filled in as they are added)."""


def declare(L):
    return L
