"""Drop-in for the row-batch helpers of InchingLiteInteger.util (util.py:563-589)."""
from .graph import flatten_partition_tree, partition_tree


def GetPartitionTree(iteratorA, maxleafsize=108):
    return partition_tree(len(iteratorA), maxleafsize)


def FlattenPartitionTree(nested):
    return flatten_partition_tree(nested)
